"""
The int64 field and NTT (zkgpu.field_gpu, zkgpu.ntt_gpu) without a GPU: the
oracle against the reference's own outputs (tests/golden/field64.json), the
argument validation the reference's tests/test_field_gpu.py:150-175 and
tests/test_ntt.py:279-282 hold, which runs before any device work, and the
loud failure when no CUDA device is present.
"""

from __future__ import annotations

import hashlib
import random

import numpy as np
import pytest

from conftest import golden
from oracle import pyoracle as po
from zkgpu import field_gpu
from zkgpu.curve import R as BN254_R
from zkgpu.ntt_gpu import ntt_gpu


def i64_digest(values) -> str:
    return hashlib.sha256(np.asarray(values, dtype="<i8").tobytes()).hexdigest()


def ntt_cases():
    for mod, per in golden("field64.json")["ntt"].items():
        for n, entry in per.items():
            yield pytest.param(int(mod), n, entry, id=f"{mod}-{n}")


@pytest.mark.parametrize("mod,n,entry", list(ntt_cases()))
def test_oracle_ntt_matches_reference(mod, n, entry):
    if n == "unreduced":
        a = entry["input"]
    else:
        rng = random.Random(int(n))
        a = [rng.randrange(mod) for _ in range(int(n))]
    fwd, inv = po.ntt(a, mod), po.ntt(a, mod, invert=True)
    if "fwd" in entry:
        assert fwd == entry["fwd"] and inv == entry["inv"]
    else:
        assert i64_digest(fwd) == entry["fwd_sha256"] and i64_digest(inv) == entry["inv_sha256"]
    if mod < 2**32:
        assert po.ntt_np(a, mod).tolist() == fwd
        assert po.ntt_np(a, mod, invert=True).tolist() == inv


def test_golden_ops_are_exact_integers():
    """The fixture's answers (the reference's fallback) equal exact integer arithmetic."""
    for mod, e in golden("field64.json")["ops"].items():
        m = int(mod)
        assert e["mul"] == [x * y % m for x, y in zip(e["a"], e["b"], strict=True)]
        assert e["add"] == [(x + y) % m for x, y in zip(e["a"], e["b"], strict=True)]
        for k, got in e["pow"].items():
            base = e["inv_bases"] if int(k) < 0 else e["b"]
            assert got == [pow(x, int(k), m) for x in base]


@pytest.mark.parametrize("mod", [0, 1, -7, 2**63])
def test_rejects_modulus_outside_int64_range(mod):
    x = np.array([1, 2], dtype=np.int64)
    for f in (field_gpu.gpu_batch_mul, field_gpu.gpu_batch_add):
        with pytest.raises(ValueError, match="2 <= mod < 2"):
            f(x, x, mod)
    with pytest.raises(ValueError, match="2 <= mod < 2"):
        field_gpu.gpu_batch_pow(x, 2, mod)


def test_rejects_non_integer_arguments():
    ints = np.array([1, 2], dtype=np.int64)
    floats = np.array([1.5, 2.0])
    with pytest.raises(TypeError):
        field_gpu.gpu_batch_mul(ints, ints, 7.0)
    with pytest.raises(TypeError, match="integer array"):
        field_gpu.gpu_batch_mul(floats, ints, 7)
    with pytest.raises(TypeError, match="integer array"):
        field_gpu.gpu_batch_add(ints, floats, 7)
    with pytest.raises(TypeError, match="integer array"):
        field_gpu.gpu_batch_pow(floats, 2, 7)
    with pytest.raises(TypeError):
        field_gpu.gpu_batch_pow(ints, 2.0, 7)


def test_torch_float_tensors_are_refused():
    torch = pytest.importorskip("torch")
    with pytest.raises(TypeError, match="integer array"):
        field_gpu.gpu_batch_mul(torch.ones(2), torch.ones(2, dtype=torch.int64), 7)
    with pytest.raises(TypeError, match="integer array"):
        field_gpu.gpu_batch_add(torch.ones(2, dtype=torch.bool), torch.ones(2, dtype=torch.int64), 7)


def test_ntt_rejects_modulus_beyond_int64():
    with pytest.raises(ValueError, match="below 2\\^63"):
        ntt_gpu(np.arange(4, dtype=np.int64), BN254_R)


def test_no_cpu_fallback_without_a_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    x = np.array([1, 2], dtype=np.int64)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        field_gpu.gpu_batch_mul(x, x, 7)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        ntt_gpu(x, 998_244_353)


def test_ntt64_c_abi_refuses_overlapping_buffers():
    """zkb_ntt64 gathers its input in bit-reversed order, so in and out must not overlap: the
    C ABI refuses it before any device work (addresses only; skipped where a GPU is visible,
    so that no kernel could ever see these stand-in pointers)."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    from zkgpu import _native

    lib = _native.lib()
    base = 1 << 20
    for out in (base, base + 8, base + 24):
        rc = lib.zkb_ntt64(base, out, 4, 998_244_353, 911_660_635, 0, base + 4096, 1 << 16, None)
        assert rc == 1 and "overlap" in _native.last_error()
