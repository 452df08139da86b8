"""
zkgpu.field256_gpu on the GPU, bit-exact against the reference's golden rows
and the oracle (the reference's tests/test_field256_gpu.py, case by case,
plus the configs' sizes: NTT 2^12, 2^16, 2^20 against the reference's own
outputs, 2^22 and 2^24 against the C oracle).
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
from zkgpu.curve import P, R
from zkgpu.field256_gpu import BN254_FQ, BN254_FR, Field256

pytestmark = pytest.mark.gpu

FIELDS = [
    pytest.param(BN254_FR, id="bn254-r"),
    pytest.param(BN254_FQ, id="bn254-p"),
    pytest.param(Field256(2**255 - 19), id="2^255-19"),
    pytest.param(Field256(3), id="3"),
    pytest.param(Field256(2**64 + 13), id="2^64+13"),
]

# BLS12-381's scalar field: a prime below 2^255 with 2-adicity 32, to run the
# NTT through the runtime-modulus kernels
BLS12_381_R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001


def rows_ints(t) -> list[int]:
    return wl.rows_to_ints(t.cpu().numpy())


def digest(t) -> str:
    return hashlib.sha256(np.ascontiguousarray(t.cpu().numpy(), dtype="<u8").tobytes()).hexdigest()


def operands(p: int, seed: int):
    """Every pair of carry-sensitive edge values, plus random residues (reference test :46-52)."""
    edge = sorted({e % p for e in (0, 1, 2, p - 1, p - 2, p // 2, 2**64 - 1, 2**128 - 1, 2**192 - 1)})
    rng = random.Random(seed)
    a = [x for x in edge for _ in edge] + [rng.randrange(p) for _ in range(500)]
    b = edge * len(edge) + [rng.randrange(p) for _ in range(500)]
    return a, b


def test_rows_hold_montgomery_form():
    import torch

    rows = BN254_FR.from_ints([1, 0])
    assert rows.dtype == torch.uint64 and tuple(rows.shape) == (2, 4) and rows.is_cuda
    r_mod = 0x0E0A77C19A07DF2F666EA36F7879462E36FC76959F60CD29AC96341C4FFFFFFB
    assert rows.cpu().tolist()[0] == [(r_mod >> (64 * j)) & (2**64 - 1) for j in range(4)]
    assert rows.cpu().tolist()[1] == [0, 0, 0, 0]


@pytest.mark.parametrize("modulus", list(golden("field.json").keys()))
def test_rows_are_the_references_rows(modulus):
    """from_ints, mul, add and sub produce the reference's exact Montgomery rows."""
    g = golden("field.json")[modulus]
    F = Field256(h(modulus))
    A, B = F.from_ints(hs(g["a"])), F.from_ints(hs(g["b"]))
    assert rows_ints(A) == hs(g["a_rows"])
    assert rows_ints(F.mul(A, B)) == hs(g["mul_rows"])
    assert rows_ints(F.add(A, B)) == hs(g["add_rows"])
    assert rows_ints(F.sub(A, B)) == hs(g["sub_rows"])


@pytest.mark.parametrize("field", FIELDS)
def test_round_trip(field):
    p = field.modulus
    values = [0, 1, p - 1, p, p + 1, -1, -p, 3 * p + 5, 2**256 + 9]
    assert field.to_ints(field.from_ints(values)) == [v % p for v in values]


@pytest.mark.parametrize("field", FIELDS)
@pytest.mark.parametrize("op", ["mul", "add", "sub"])
def test_ops_match_python(field, op):
    p = field.modulus
    a, b = operands(p, {"mul": 1, "add": 2, "sub": 3}[op])
    got = field.to_ints(getattr(field, op)(field.from_ints(a), field.from_ints(b)))
    fn = {"mul": lambda x, y: x * y, "add": lambda x, y: x + y, "sub": lambda x, y: x - y}[op]
    assert got == [fn(x, y) % p for x, y in zip(a, b, strict=True)]


@pytest.mark.parametrize("field", FIELDS)
def test_squaring_matches_python(field):
    """mul(x, x) on the same rows takes the squaring path (separated operand scanning): exact
    against Python integers on random values and the carry-heavy edges, broadcast row included."""
    F = field
    p = F.modulus
    rng = random.Random(p % 997)
    values = [0, 1, 2, p - 1, p - 2, (p - 1) // 2, (p + 1) // 2] + [rng.randrange(p) for _ in range(4000)]
    values += [min(p - 1, (1 << k) - 1) for k in range(1, p.bit_length() + 1)]
    rows = F.from_ints(values)
    assert F.to_ints(F.mul(rows, rows)) == [v * v % p for v in values]
    one = F.from_ints([p - 1])
    assert F.to_ints(F.mul(one, one)) == [1]


def extreme_values(p: int, seed: int) -> list[int]:
    """Canonical values whose 32-bit words push the product's carry chains to their ends: p - 1 and
    its neighbours, words of all ones, p minus powers of 2^32, and values whose words are each 0,
    0xffffffff or random (the top bits cleared to stay below p, so the word pattern survives)."""
    vals = {0, 1, 2, p - 1, p - 2, p - 3}
    for k in range(1, 9):
        vals.add(min(p - 1, (1 << (32 * k)) - 1))
        vals.add(p - (1 << (32 * (k - 1))))
        vals.add(p - 1 - ((1 << (32 * (k - 1))) - 1))
    rng = random.Random(seed)
    keep = (1 << (p.bit_length() - 1)) - 1
    while len(vals) < 72:
        v = 0
        for w in range(8):
            v |= rng.choice((0, 0xFFFFFFFF, 0xFFFFFFFF, rng.getrandbits(32))) << (32 * w)
        vals.add(v if v < p else v & keep)
    return sorted(vals)


@pytest.mark.parametrize("field", FIELDS[:3])
def test_raw_rows_with_extreme_words(field):
    """The Montgomery product and squaring on raw rows (no conversion, so the kernel sees these exact
    words): every pair of the extreme values gives a b 2^-256 mod p, every square a^2 2^-256 mod p."""
    from zkgpu import _rows

    p = field.modulus
    vals = extreme_values(p, p % 1009)
    a = [x for x in vals for _ in vals]
    b = vals * len(vals)
    rinv = pow(2**256, -1, p)
    A = _rows.upload(_rows.ints_to_limbs(a))
    B = _rows.upload(_rows.ints_to_limbs(b))
    got = _rows.limbs_to_ints(_rows.download(field.mul(A, B)))
    assert got == [x * y * rinv % p for x, y in zip(a, b, strict=True)]
    S = _rows.upload(_rows.ints_to_limbs(vals))
    got = _rows.limbs_to_ints(_rows.download(field.mul(S, S)))  # the same rows: the squaring path
    assert got == [x * x * rinv % p for x in vals]


def test_operations_compose():
    F, p = BN254_FQ, P
    a, b = operands(p, 4)
    A, B = F.from_ints(a), F.from_ints(b)
    lhs = F.to_ints(F.mul(F.add(A, B), F.sub(A, B)))
    rhs = F.to_ints(F.sub(F.mul(A, A), F.mul(B, B)))
    assert lhs == rhs == [(x * x - y * y) % p for x, y in zip(a, b, strict=True)]


def test_large_batch_matches_c_oracle():
    """2^20 rows (32 MiB per operand, the reference's largest mul benchmark) against the C oracle."""
    n = 1 << 20
    a, b = wl.uniform_fr(41, n), wl.uniform_fr(42, n)
    A, B = BN254_FR.to_montgomery(a), BN254_FR.to_montgomery(b)
    ca, cb = co.to_mont(co.FR, a), co.to_mont(co.FR, b)
    assert np.array_equal(A.cpu().numpy(), ca)
    assert np.array_equal(BN254_FR.mul(A, B).cpu().numpy(), co.field_op("mul", co.FR, ca, cb))
    assert np.array_equal(BN254_FR.sub(A, B).cpu().numpy(), co.field_op("sub", co.FR, ca, cb))
    assert np.array_equal(BN254_FR.from_montgomery(A).cpu().numpy(), a)


def test_single_row_broadcasts_on_either_side():
    F, p = BN254_FR, R
    values = [3, 5, p - 1, 0]
    rows, c = F.from_ints(values), F.from_ints([p - 2])
    assert F.to_ints(F.mul(rows, c)) == [v * (p - 2) % p for v in values]
    assert F.to_ints(F.sub(c, rows)) == [(p - 2 - v) % p for v in values]
    assert F.to_ints(F.add(c, c)) == [(2 * (p - 2)) % p]


def test_empty_batches():
    F = BN254_FR
    empty = F.from_ints([])
    assert tuple(empty.shape) == (0, 4)
    assert F.to_ints(F.mul(empty, empty)) == []
    assert F.to_ints(F.add(empty, F.from_ints([7]))) == []


def test_numpy_and_dlpack_inputs_are_accepted():
    import torch

    rows = BN254_FR.from_ints([5, 6, 7])
    host = rows.cpu().numpy()
    assert BN254_FR.to_ints(BN254_FR.mul(host, rows)) == [25, 36, 49]
    assert BN254_FR.to_ints(BN254_FR.add(torch.utils.dlpack.from_dlpack(rows), rows)) == [10, 12, 14]


def test_self_test_passes():
    for field in (BN254_FR, BN254_FQ, Field256(2**255 - 19), Field256(BLS12_381_R)):
        field.compile()


# ------------------------------------------------------------------
# NTT
# ------------------------------------------------------------------


@pytest.mark.parametrize("n", [1, 2, 4, 8, 64, 1024, 4096])
def test_ntt_matches_the_references(n):
    """Forward, inverse and both coset transforms, against the reference's outputs."""
    entry = golden("ntt.json")["small"][str(n)]
    rng = random.Random(n)
    a = [rng.randrange(R) for _ in range(n)]
    rows = BN254_FR.from_ints(a)
    g = entry["coset_offset"]
    outs = {
        "fwd": BN254_FR.ntt(rows),
        "inv": BN254_FR.ntt(rows, invert=True),
        "coset_fwd": BN254_FR.ntt(rows, coset=g),
        "coset_inv": BN254_FR.ntt(rows, invert=True, coset=g),
    }
    for key, out in outs.items():
        if key in entry:
            assert BN254_FR.to_ints(out) == hs(entry[key]), key
        else:
            assert digest(out) == entry[key + "_sha256"], key


@pytest.mark.parametrize("n", ["65536", "1048576"])
def test_large_ntt_matches_the_references(n):
    """2^16 and 2^20 (config 2's NTT size), forward / inverse / coset, by digest of the reference's rows."""
    entry = golden("ntt.json")["large"].get(n)
    if entry is None:
        pytest.skip("fixture generated with --quick")
    rows = BN254_FR.to_montgomery(wl.uniform_fr(entry["seed"], int(n)))
    assert digest(rows) == entry["input_sha256"]
    assert digest(BN254_FR.ntt(rows)) == entry["fwd_sha256"]
    assert digest(BN254_FR.ntt(rows, invert=True)) == entry["inv_sha256"]
    if "coset_fwd_sha256" in entry:
        assert digest(BN254_FR.ntt(rows, coset=5)) == entry["coset_fwd_sha256"]
        assert digest(BN254_FR.ntt(rows, coset=5, invert=True)) == entry["coset_inv_sha256"]


@pytest.mark.parametrize("log_n", [13, 17, 22])
def test_ntt_matches_c_oracle_between_fixture_sizes(log_n):
    """Sizes with uneven pass splits (13 = 7 + 6) and up to 2^22, against the C oracle."""
    n = 1 << log_n
    rows_h = co.to_mont(co.FR, wl.uniform_fr(50 + log_n, n))
    rows = BN254_FR.to_montgomery(wl.uniform_fr(50 + log_n, n))
    threads = os.cpu_count() or 1
    for invert in (False, True):
        for coset in (None, 5):
            want = co.ntt(rows_h, invert=invert, coset=coset, threads=threads)
            got = BN254_FR.ntt(rows, invert=invert, coset=coset).cpu().numpy()
            assert np.array_equal(got, want), (invert, coset)


@pytest.mark.parametrize(
    "knobs",
    [
        {"ntt.max_log_radix": 8},  # three passes at 2^20 and above
        {"ntt.max_log_radix": 12},  # two passes up to 2^24 (4096-row tiles of 512 threads there)
        {"ntt.max_log_radix": 12, "ntt.cta_log_elems": 10},  # 1024-row tiles of 256 threads
        {"ntt.max_log_radix": 9, "ntt.cta_log_elems": 9, "ntt.threads": 64},
        {"ntt.cta_log_elems": 12, "ntt.threads": 128},
        {"ntt.cta_log_elems": 10, "ntt.threads": 512},
        {"ntt.full_table_mb": 0},  # two-level twiddle and coset tables only
        {"ntt.max_log_radix": 8, "ntt.full_table_mb": 1},  # expanded tables for the small sizes only
        {"ntt.tma": 0},  # per-thread gathers instead of the TMA-fed persistent passes
        {"ntt.tma": 0, "ntt.max_log_radix": 12},
    ],
)
def test_ntt_pass_plans_give_the_same_rows(knobs):
    """Every pass split, tile size and block size the tuning knobs allow computes the same rows
    (against the reference's digests at 2^16 and 2^20, and the C oracle at 2^13 and 2^21)."""
    from zkgpu import _native

    try:
        for k, v in knobs.items():
            _native.tune_set(k, v)
        for n in ("65536", "1048576"):
            entry = golden("ntt.json")["large"].get(n)
            if entry is None:
                continue
            rows = BN254_FR.to_montgomery(wl.uniform_fr(entry["seed"], int(n)))
            assert digest(BN254_FR.ntt(rows)) == entry["fwd_sha256"], n
            assert digest(BN254_FR.ntt(rows, invert=True)) == entry["inv_sha256"], n
            if "coset_fwd_sha256" in entry:
                assert digest(BN254_FR.ntt(rows, coset=5)) == entry["coset_fwd_sha256"], n
                assert digest(BN254_FR.ntt(rows, coset=5, invert=True)) == entry["coset_inv_sha256"], n
        for log_n in (13, 21):
            n = 1 << log_n
            rows = BN254_FR.to_montgomery(wl.uniform_fr(60 + log_n, n))
            host = co.to_mont(co.FR, wl.uniform_fr(60 + log_n, n))
            for invert, coset in ((False, None), (True, 5)):
                want = co.ntt(host, invert=invert, coset=coset, threads=os.cpu_count() or 1)
                got = BN254_FR.ntt(rows, invert=invert, coset=coset).cpu().numpy()
                assert np.array_equal(got, want), (log_n, invert, coset)
    finally:
        _native.tune_set("ntt.max_log_radix", 0)
        _native.tune_set("ntt.cta_log_elems", 0)
        _native.tune_set("ntt.threads", 0)
        _native.tune_set("ntt.full_table_mb", 4096)
        _native.tune_set("ntt.tma", 1)


@pytest.mark.parametrize("cta_log", [9, 10, 11, 12])
def test_tma_passes_equal_gather_passes_at_every_size(cta_log):
    """The TMA-fed persistent passes (decimation in frequency over natural-order tiles) give the
    rows of the per-thread gather passes (decimation in time over bit-reversed gathers) for
    every size 2^2..2^22, forward / inverse / coset, at every tile size (two buffers up to
    2048-row tiles, one at 4096); no tile's TMA wait gives up."""
    from zkgpu import _native

    lib = _native.lib()
    before = lib.zkb_ntt_wait_timeouts()
    try:
        _native.tune_set("ntt.cta_log_elems", cta_log)
        for log_n in range(2, 23):
            n = 1 << log_n
            rows = BN254_FR.to_montgomery(wl.uniform_fr(300 + log_n, n))
            for invert, coset in ((False, None), (True, None), (False, 5), (True, 7)):
                _native.tune_set("ntt.tma", 1)
                got = BN254_FR.ntt(rows, invert=invert, coset=coset)
                _native.tune_set("ntt.tma", 0)
                want = BN254_FR.ntt(rows, invert=invert, coset=coset)
                assert bool((got == want).all()), (log_n, invert, coset)
    finally:
        _native.tune_set("ntt.tma", 1)
        _native.tune_set("ntt.cta_log_elems", 0)
    assert lib.zkb_ntt_wait_timeouts() == before == 0


@pytest.mark.parametrize("cta_log", [9, 12])
def test_lazy_reduction_passes_give_the_same_rows(cta_log):
    """TMA passes with values in [0, 2p) between rounds ("ntt.lazy" = 1) give the canonical
    passes' rows for every size 2^2..2^22, forward / inverse / coset, at both tile sizes; and at
    2^20 the rows of the C port. Inputs include 0, 1 and p - 1 (the values the lazy ranges'
    edges are made of)."""
    from zkgpu import _native

    lib = _native.lib()
    saved = _native.tune_get("ntt.lazy")
    try:
        _native.tune_set("ntt.cta_log_elems", cta_log)
        for log_n in range(2, 23):
            n = 1 << log_n
            plain = wl.uniform_fr(400 + log_n, n)
            plain[0] = (0, 0, 0, 0)
            plain[n // 2] = _native.limbs(R - 1)
            plain[n - 1] = (1, 0, 0, 0)
            rows = BN254_FR.to_montgomery(plain)
            for invert, coset in ((False, None), (True, None), (False, 5), (True, 7)):
                _native.tune_set("ntt.lazy", 1)
                got = BN254_FR.ntt(rows, invert=invert, coset=coset)
                _native.tune_set("ntt.lazy", 0)
                want = BN254_FR.ntt(rows, invert=invert, coset=coset)
                assert bool((got == want).all()), (log_n, invert, coset)
        n = 1 << 20
        plain = wl.uniform_fr(499, n)
        _native.tune_set("ntt.lazy", 1)
        got = BN254_FR.ntt(BN254_FR.to_montgomery(plain), coset=5)
        assert np.array_equal(got.cpu().numpy(), co.ntt(co.to_mont(co.FR, plain), coset=5, threads=os.cpu_count() or 1))
    finally:
        _native.tune_set("ntt.lazy", saved)
        _native.tune_set("ntt.cta_log_elems", 0)
    assert lib.zkb_ntt_wait_timeouts() == 0


def test_ntt_2_24_config_size():
    """Config 3's NTT: 2^24 elements (512 MiB), plain and coset g = 5, against the C oracle,
    plus the size-independent round trips."""
    n = 1 << 24
    plain = wl.uniform_fr(5, n)
    rows = BN254_FR.to_montgomery(plain)
    before = rows.clone()
    threads = os.cpu_count() or 1
    host = co.to_mont(co.FR, plain)
    fwd = BN254_FR.ntt(rows)
    assert np.array_equal(fwd.cpu().numpy(), co.ntt(host, threads=threads))
    cfwd = BN254_FR.ntt(rows, coset=5)
    assert np.array_equal(cfwd.cpu().numpy(), co.ntt(host, coset=5, threads=threads))
    assert bool((BN254_FR.ntt(fwd, invert=True) == before).all())
    assert bool((BN254_FR.ntt(cfwd, invert=True, coset=5) == before).all())
    assert bool((rows == before).all())  # the input is never modified


@pytest.mark.parametrize("n", [8, 256])
def test_ntt_of_x_lists_the_domain(n):
    x = [0, 1] + [0] * (n - 2)
    assert BN254_FR.to_ints(BN254_FR.ntt(BN254_FR.from_ints(x))) == hs(golden("ntt.json")["elements"][str(n)])


def test_ntt_round_trip_leaves_input_unchanged():
    rng = random.Random(9)
    a = [rng.randrange(R) for _ in range(512)]
    rows = BN254_FR.from_ints(a)
    before = rows.cpu().tolist()
    assert BN254_FR.to_ints(BN254_FR.ntt(BN254_FR.ntt(rows), invert=True)) == a
    assert rows.cpu().tolist() == before


def test_ntt_multiplies_polynomials():
    F, n = BN254_FR, 64
    rng = random.Random(5)
    a, b = [rng.randrange(R) for _ in range(n)], [rng.randrange(R) for _ in range(n)]
    product = F.ntt(F.mul(F.ntt(F.from_ints(a)), F.ntt(F.from_ints(b))), invert=True)
    expected = [0] * n
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            expected[(i + j) % n] = (expected[(i + j) % n] + x * y) % R
    assert F.to_ints(product) == expected


def test_ntt_of_nothing():
    assert tuple(BN254_FR.ntt(BN254_FR.from_ints([])).shape) == (0, 4)


@pytest.mark.parametrize("n", [2, 64, 4096, 1 << 14])
def test_ntt_over_a_runtime_modulus(n):
    """A prime other than BN254's runs the runtime-modulus kernels with the caller's root."""
    F = Field256(BLS12_381_R)
    rng = random.Random(n)
    a = [rng.randrange(BLS12_381_R) for _ in range(n)]
    rows = F.from_ints(a)
    if n <= 64:
        assert F.to_ints(F.ntt(rows)) == po.ntt(a, BLS12_381_R)
        assert F.to_ints(F.ntt(rows, invert=True, coset=7)) == po.coset_ifft(a, 7, BLS12_381_R)
    assert F.to_ints(F.ntt(F.ntt(rows, coset=7), invert=True, coset=7)) == a


def test_tiny_fields_ntt():
    """2^255 - 19 and 2^64 + 13 admit sizes 2 and 4 only; Fq admits 2."""
    for F in (Field256(2**255 - 19), Field256(2**64 + 13), BN254_FQ):
        p = F.modulus
        n = 4 if (p - 1) % 4 == 0 else 2
        a = list(range(3, 3 + n))
        assert F.to_ints(F.ntt(F.from_ints(a))) == po.ntt(a, p)
        assert F.to_ints(F.ntt(F.from_ints(a), invert=True)) == po.ntt(a, p, invert=True)
