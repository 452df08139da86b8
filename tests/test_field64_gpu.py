"""
zkgpu.field_gpu and zkgpu.ntt_gpu on the GPU, bit-exact against the
reference's own outputs (tests/golden/field64.json) and exact integers: the
cases of the reference's tests/test_field_gpu.py and tests/test_ntt.py:223-276,
plus sizes up to 2^22 against the oracle's vectorised NTT, round trips at
2^23 and 2^24, every tile shape the int64 NTT's knobs allow at small sizes,
and moduli on both sides of the Montgomery / 128-bit-remainder split.
"""

from __future__ import annotations

import hashlib
import random

import numpy as np
import pytest

from conftest import golden
from oracle import pyoracle as po
from zkgpu import field_gpu
from zkgpu.ntt_gpu import ntt_gpu

pytestmark = pytest.mark.gpu

NTT_MOD = 998_244_353
INT64_SAFE_LIMIT = 3_037_000_500
LARGEST_INT64_PRIME = 2**63 - 25
LARGE_INT64_NTT_PRIME = 2_147_483_641 * 2**32 + 1
INT64_MIN, INT64_MAX = -(2**63), 2**63 - 1
MODULI = [7, NTT_MOD, INT64_SAFE_LIMIT, INT64_SAFE_LIMIT + 1, 2**61 - 1, LARGEST_INT64_PRIME]
GPU_NTT_MODULI = [NTT_MOD, 12_289, LARGE_INT64_NTT_PRIME]


def dev(values, dtype=np.int64):
    import torch

    return torch.from_numpy(np.array(values, dtype=dtype)).cuda()


def field_elements(n: int, mod: int, seed: int) -> list[int]:
    rng = random.Random(seed)
    return [rng.randrange(mod) for _ in range(n)]


def i64_digest(t) -> str:
    return hashlib.sha256(t.cpu().numpy().astype("<i8").tobytes()).hexdigest()


# ---- element-wise ops: the reference's outputs

@pytest.mark.parametrize("mod", [int(m) for m in golden("field64.json")["ops"]])
def test_ops_match_reference_outputs(mod):
    e = golden("field64.json")["ops"][str(mod)]
    a, b = dev(e["a"]), dev(e["b"])
    assert field_gpu.gpu_batch_mul(a, b, mod).tolist() == e["mul"]
    assert field_gpu.gpu_batch_add(a, b, mod).tolist() == e["add"]
    for k, want in e["pow"].items():
        base = dev(e["inv_bases"]) if int(k) < 0 else b
        assert field_gpu.gpu_batch_pow(base, int(k), mod).tolist() == want


@pytest.mark.parametrize("mod", MODULI)
def test_batch_mul_add_match_python(mod):
    a, b = field_elements(1000, mod, 1), field_elements(1000, mod, 2)
    got = field_gpu.gpu_batch_mul(dev(a), dev(b), mod)
    assert str(got.dtype) == "torch.int64" and got.is_cuda
    assert got.tolist() == [x * y % mod for x, y in zip(a, b, strict=True)]
    assert field_gpu.gpu_batch_add(dev(a), dev(b), mod).tolist() == [(x + y) % mod for x, y in zip(a, b, strict=True)]


@pytest.mark.parametrize("mod", [INT64_SAFE_LIMIT, INT64_SAFE_LIMIT + 1, LARGEST_INT64_PRIME, 2**62, 2**63 - 2])
def test_extreme_residues(mod):
    a = [mod - 1, mod - 1, mod - 2, 0, 1]
    b = [mod - 1, 1, mod - 1, mod - 1, mod - 1]
    assert field_gpu.gpu_batch_mul(dev(a), dev(b), mod).tolist() == [x * y % mod for x, y in zip(a, b, strict=True)]
    assert field_gpu.gpu_batch_add(dev(a), dev(b), mod).tolist() == [(x + y) % mod for x, y in zip(a, b, strict=True)]


@pytest.mark.parametrize("mod", [2, 4, 2**32, 2**40 + 2, 6 * 10**18])
def test_even_moduli(mod):
    """Even moduli take the exact 128-bit remainder instead of Montgomery products."""
    rng = random.Random(mod)
    a = [rng.randrange(INT64_MIN, INT64_MAX) for _ in range(500)]
    b = [rng.randrange(INT64_MIN, INT64_MAX) for _ in range(500)]
    assert field_gpu.gpu_batch_mul(dev(a), dev(b), mod).tolist() == [x * y % mod for x, y in zip(a, b, strict=True)]
    assert field_gpu.gpu_batch_add(dev(a), dev(b), mod).tolist() == [(x + y) % mod for x, y in zip(a, b, strict=True)]
    assert field_gpu.gpu_batch_pow(dev(a), 12345, mod).tolist() == [pow(x, 12345, mod) for x in a]


@pytest.mark.parametrize("exp", [0, 1, 2, 65537, NTT_MOD - 2])
def test_batch_pow_matches_python(exp):
    bases = field_elements(256, NTT_MOD, 5)
    assert field_gpu.gpu_batch_pow(dev(bases), exp, NTT_MOD).tolist() == [pow(x, exp, NTT_MOD) for x in bases]


@pytest.mark.parametrize("exp", [3, 2**61 - 3, 2**200 + 7])
def test_batch_pow_large_modulus(exp):
    mod = 2**61 - 1
    bases = field_elements(64, mod, 6)
    assert field_gpu.gpu_batch_pow(dev(bases), exp, mod).tolist() == [pow(x, exp, mod) for x in bases]


@pytest.mark.parametrize("mod", [7, LARGEST_INT64_PRIME])
def test_unreduced_and_negative_inputs_reduce_into_field(mod):
    a = [-3, -10, INT64_MAX, INT64_MIN, 12, 0]
    b = [5, 1, INT64_MAX, INT64_MIN, -12, -1]
    assert field_gpu.gpu_batch_mul(dev(a), dev(b), mod).tolist() == [x * y % mod for x, y in zip(a, b, strict=True)]
    assert field_gpu.gpu_batch_add(dev(a), dev(b), mod).tolist() == [(x + y) % mod for x, y in zip(a, b, strict=True)]
    assert field_gpu.gpu_batch_pow(dev(a), 3, mod).tolist() == [pow(x, 3, mod) for x in a]


def test_narrow_integer_dtypes_are_widened():
    values = dev([NTT_MOD - 1, 3], dtype=np.int32)
    assert field_gpu.gpu_batch_mul(values, values, NTT_MOD).tolist() == [pow(NTT_MOD - 1, 2, NTT_MOD), 9]
    assert field_gpu.gpu_batch_pow(values, 2, 2**61 - 1).tolist() == [(NTT_MOD - 1) ** 2, 9]
    # host NumPy arrays and lists are accepted too
    assert field_gpu.gpu_batch_add(np.array([5], dtype=np.uint8), [4], 7).tolist() == [2]


def test_broadcasting():
    a = dev([[1, 2, 3], [4, 5, 6]])
    w = dev([10, 20, 30])
    assert field_gpu.gpu_batch_mul(a, w, 7).tolist() == [[10 % 7, 40 % 7, 90 % 7], [40 % 7, 100 % 7, 180 % 7]]
    assert field_gpu.gpu_batch_add(a, dev(3), 7).tolist() == [[4, 5, 6], [0, 1, 2]]


def test_non_contiguous_inputs():
    a = dev(list(range(20)))[::2]
    assert field_gpu.gpu_batch_mul(a, a, 11).tolist() == [(x * x) % 11 for x in range(0, 20, 2)]


def test_empty_inputs():
    e = dev([])
    assert field_gpu.gpu_batch_mul(e, e, 7).numel() == 0
    assert field_gpu.gpu_batch_pow(e, -1, 7).numel() == 0
    assert ntt_gpu(e, NTT_MOD).numel() == 0


def test_batch_pow_negative_exponent_is_inverse():
    for exp in (-1, -3):
        assert field_gpu.gpu_batch_pow(dev([3, 5, 6]), exp, 7).tolist() == [pow(x, exp, 7) for x in (3, 5, 6)]


def test_batch_pow_negative_exponent_rejects_zero():
    with pytest.raises(ValueError, match="not invertible"):
        field_gpu.gpu_batch_pow(dev([3, 7]), -1, 7)


def test_large_batch_against_numpy():
    """2^24 elements: every grid-stride path, checked against NumPy (mod < 2^32: products fit uint64)."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(7)
    a = torch.randint(INT64_MIN, INT64_MAX, (1 << 24,), device="cuda", generator=g)
    b = torch.randint(INT64_MIN, INT64_MAX, (1 << 24,), device="cuda", generator=g)
    an, bn = np.mod(a.cpu().numpy(), NTT_MOD).astype(np.uint64), np.mod(b.cpu().numpy(), NTT_MOD).astype(np.uint64)
    m = np.uint64(NTT_MOD)
    assert np.array_equal(field_gpu.gpu_batch_mul(a, b, NTT_MOD).cpu().numpy(), (an * bn % m).astype(np.int64))
    assert np.array_equal(field_gpu.gpu_batch_add(a, b, NTT_MOD).cpu().numpy(), ((an + bn) % m).astype(np.int64))


# ---- NTT

def ntt_golden_cases():
    for mod, per in golden("field64.json")["ntt"].items():
        for n, entry in per.items():
            yield pytest.param(int(mod), n, entry, id=f"{mod}-{n}")


@pytest.mark.parametrize("mod,n,entry", list(ntt_golden_cases()))
def test_ntt_matches_reference_outputs(mod, n, entry):
    if n == "unreduced":
        a = entry["input"]
    else:
        rng = random.Random(int(n))
        a = [rng.randrange(mod) for _ in range(int(n))]
    fwd, inv = ntt_gpu(dev(a), mod), ntt_gpu(dev(a), mod, invert=True)
    if "fwd" in entry:
        assert fwd.tolist() == entry["fwd"] and inv.tolist() == entry["inv"]
    else:
        assert i64_digest(fwd) == entry["fwd_sha256"] and i64_digest(inv) == entry["inv_sha256"]


@pytest.mark.parametrize("mod", GPU_NTT_MODULI)
@pytest.mark.parametrize("n", [1, 2, 8, 256, 1 << 12])
def test_ntt_matches_cpu(n, mod):
    rng = random.Random(n)
    a = [rng.randrange(mod) for _ in range(n)]
    assert ntt_gpu(dev(a), mod).tolist() == po.ntt(a, mod)


@pytest.mark.parametrize("log_n", [10, 11, 12, 13, 14, 16, 20, 22])
def test_ntt_matches_oracle_sizes(log_n):
    """Sizes around the shared-memory tile (2^11) and up to 2^22, against the oracle's NumPy NTT."""
    import torch

    n = 1 << log_n
    g = torch.Generator(device="cuda").manual_seed(log_n)
    a = torch.randint(INT64_MIN, INT64_MAX, (n,), device="cuda", generator=g)
    host = a.cpu().numpy()
    assert np.array_equal(ntt_gpu(a, NTT_MOD).cpu().numpy(), po.ntt_np(host, NTT_MOD))
    assert np.array_equal(ntt_gpu(a, NTT_MOD, invert=True).cpu().numpy(), po.ntt_np(host, NTT_MOD, invert=True))


TILE_SHAPES = [(0, 4, 1, 2), (2, 10, 3, 9), (3, 9, 4, 8), (5, 8, 5, 8), (6, 7, 6, 7), (6, 10, 6, 10), (1, 5, 2, 3)]


@pytest.mark.parametrize("shape", TILE_SHAPES, ids=str)
def test_ntt_tile_shapes(shape):
    """Every pass plan the knobs ntt64.* give (first-pass columns and stages, later-pass columns and
    stages) against the oracle, 2^0 .. 2^16, forward and inverse."""
    import torch

    from zkgpu import _native

    keys = ("ntt64.first_col_log", "ntt64.first_max_k", "ntt64.col_log", "ntt64.max_k")
    try:
        for k, v in zip(keys, shape):
            _native.tune_set(k, v)
        for log_n in range(17):
            rng = np.random.default_rng(log_n)
            a = rng.integers(INT64_MIN, INT64_MAX, 1 << log_n, endpoint=True)
            x = torch.from_numpy(a).cuda()
            assert np.array_equal(ntt_gpu(x, NTT_MOD).cpu().numpy(), po.ntt_np(a, NTT_MOD)), log_n
            assert np.array_equal(ntt_gpu(x, NTT_MOD, invert=True).cpu().numpy(),
                                  po.ntt_np(a, NTT_MOD, invert=True)), log_n
    finally:
        for k, v in zip(keys, (-1, 0, 0, 0)):
            _native.tune_set(k, v)


@pytest.mark.parametrize("mod", GPU_NTT_MODULI)
def test_ntt_inverse_roundtrip(mod):
    rng = random.Random(55)
    a = [rng.randrange(mod) for _ in range(1024)]
    assert ntt_gpu(ntt_gpu(dev(a), mod), mod, invert=True).tolist() == a


@pytest.mark.parametrize("mod,log_n", [(NTT_MOD, 23), (LARGE_INT64_NTT_PRIME, 24)])
def test_ntt_roundtrip_and_linearity_large(mod, log_n):
    """Size-independent properties at the largest sizes: inverse(forward(a)) = a, NTT(a + b) = NTT(a) + NTT(b)."""
    import torch

    n = 1 << log_n
    g = torch.Generator(device="cuda").manual_seed(24)
    a = torch.randint(0, min(mod, INT64_MAX), (n,), device="cuda", generator=g) % mod
    b = torch.randint(0, min(mod, INT64_MAX), (n,), device="cuda", generator=g) % mod
    fa = ntt_gpu(a, mod)
    assert torch.equal(ntt_gpu(fa, mod, invert=True), a)
    lhs = ntt_gpu(field_gpu.gpu_batch_add(a, b, mod), mod)
    assert torch.equal(lhs, field_gpu.gpu_batch_add(fa, ntt_gpu(b, mod), mod))


def test_ntt_repeated_calls_agree():
    import torch

    a = torch.arange(4096, dtype=torch.int64, device="cuda")
    first = ntt_gpu(a, NTT_MOD).tolist()
    assert ntt_gpu(a, NTT_MOD).tolist() == first
    assert a.tolist() == list(range(4096))


def test_ntt_single_element_is_reduced():
    assert ntt_gpu(dev([NTT_MOD + 5]), NTT_MOD).tolist() == [5]


def test_ntt_validates_like_the_cpu_ntt():
    import torch

    with pytest.raises(ValueError, match="odd prime"):
        ntt_gpu(torch.arange(4, device="cuda"), 21)
    with pytest.raises(ValueError, match="power of 2"):
        ntt_gpu(torch.arange(3, device="cuda"), NTT_MOD)
    with pytest.raises(ValueError, match="not supported"):
        ntt_gpu(torch.arange(1 << 13, device="cuda"), 12_289)
