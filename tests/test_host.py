"""
Host-side logic that needs no GPU: argument validation and error types (the
reference's, raised before any device work), Montgomery constants, the C
ABI's exports and its host-only entry points, roots of unity, and the
no-fallback rule (device operations raise RuntimeError without a GPU).
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, golden, h, hs
from zkgpu import _native, curve_gpu, msm_gpu, roots
from zkgpu.curve import G, P, Point, R
from zkgpu.field256_gpu import BN254_FQ, BN254_FR, Field256

HEADER = ROOT / "include" / "zkb200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w]+\*?\s+\*?(zkb_\w+)\s*\(", text, re.M)))


# ------------------------------------------------------------------
# The C ABI
# ------------------------------------------------------------------


def test_header_declares_the_abi():
    names = declared_functions()
    for name in ("zkb_field_mul", "zkb_ntt", "zkb_g1_add", "zkb_msm", "zkb_last_error"):
        assert name in names
    assert set(names) == set(_native.SIGNATURES), "ctypes signatures and header disagree"


def test_library_loads_and_exports_every_declared_symbol():
    lib = _native.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.zkb_version() >= 100


@pytest.mark.parametrize("modulus", list(golden("field.json").keys()))
def test_zkb_field_init_computes_the_reference_constants(modulus):
    g = golden("field.json")[modulus]
    p = h(modulus)
    f = _native.make_field(p)
    as_int = lambda arr: sum(int(arr[j]) << (64 * j) for j in range(4))  # noqa: E731
    assert as_int(f.modulus) == p
    assert as_int(f.one) == 2**256 % p
    assert as_int(f.r2) == h(g["r2"])
    assert f.ninv == h(g["n_inv"])
    expected_kind = {R: _native.FIELD_BN254_FR, P: _native.FIELD_BN254_FQ}.get(p, _native.FIELD_GENERIC)
    assert f.kind == expected_kind


@pytest.mark.parametrize("modulus", [2, 1, 0, 2**64, 2**255 + 1, 2**256 - 189])
def test_zkb_field_init_rejects_bad_moduli(modulus):
    f = _native.ZkbField()
    status = _native.lib().zkb_field_init(ctypes.byref(f), _native.u64_array(_native.limbs(modulus % 2**256)))
    assert status == _native.ZKB_EINVAL
    assert "odd and in [3, 2^255)" in _native.last_error()


def test_status_codes_map_to_reference_exceptions():
    with pytest.raises(ValueError):
        _native.check(_native.ZKB_EINVAL)
    with pytest.raises(TypeError):
        _native.check(_native.ZKB_ETYPE)
    with pytest.raises(RuntimeError):
        _native.check(_native.ZKB_ECUDA)
    _native.check(_native.ZKB_OK)


def test_host_only_queries():
    lib = _native.lib()
    assert lib.zkb_ntt_workspace_bytes(512) == 0  # one pass, no intermediate rows
    assert lib.zkb_ntt_workspace_bytes(4096) == 4096 * 32  # split in two passes from 2^10 on
    assert lib.zkb_ntt_workspace_bytes(1 << 20) == 32 << 20
    # default window: argmin of windows * (20 n + 42 * 2^(w-1)): signed digits over
    # the two 127-bit GLV halves, ceil(128 / w) windows
    def model(n):
        best = min(range(1, 17), key=lambda w: (-(-128 // w)) * (20 * n + 42 * 2 ** (w - 1)))
        return best if n > 1 else 1
    for n in (1, 100, 2**12, 2**16, 2**20, 2**22):
        assert lib.zkb_msm_default_window(n) == model(n), n


def test_tuning_knobs_validate_and_plan_the_workspace():
    defaults = {"msm.pairs_per_thread": 0, "msm.slots_per_thread": 8, "msm.reduce_log_segment": 4, "msm.call_pairs_cap": 16, "msm.sort": 1,
                "ntt.max_log_radix": 0, "ntt.cta_log_elems": 0, "ntt.threads": 0, "ntt.full_table_mb": 4096,
                "ntt64.first_col_log": -1, "ntt64.first_max_k": 0, "ntt64.col_log": 0, "ntt64.max_k": 0}
    assert {k: _native.tune_get(k) for k in defaults} == defaults
    with pytest.raises(ValueError, match="unknown tuning knob"):
        _native.tune_set("ntt.bogus", 1)
    with pytest.raises(ValueError, match="0..12"):
        _native.tune_set("ntt.max_log_radix", 13)
    lib = _native.lib()
    try:
        # at most 8 bits per pass: 2^9 rows no longer fit one pass
        _native.tune_set("ntt.max_log_radix", 8)
        assert lib.zkb_ntt_workspace_bytes(1 << 20) == 32 << 20
        assert lib.zkb_ntt_workspace_bytes(512) == 512 * 32
        assert lib.zkb_ntt_workspace_bytes(256) == 0
    finally:
        _native.tune_set("ntt.max_log_radix", 0)
    assert lib.zkb_ntt_workspace_bytes(512) == 0


def test_batch_entry_points_validate_on_the_host():
    lib = _native.lib()
    jobs = (_native.ZkbNttJob * 65)()
    for j in range(65):
        jobs[j].n = 8
    # counters (256 B) + 192 pass counters, then 2^12 rows of intermediate storage
    jobs[0].n, jobs[1].n = 4096, 8
    assert lib.zkb_ntt_batch_workspace_bytes(jobs, 2) == 1024 + 4096 * 32
    assert lib.zkb_ntt_batch_workspace_bytes(jobs, 65) == 0
    assert "0..64" in _native.last_error()
    fr, fq = _native.make_field(R), _native.make_field(P)
    assert lib.zkb_ntt_batch(ctypes.byref(fq), jobs, 2, None, 0, None, None) == _native.ZKB_EINVAL
    assert "BN254 Fr" in _native.last_error()
    jobs[1].n = 6
    assert lib.zkb_ntt_batch(ctypes.byref(fr), jobs, 2, None, 0, None, None) == _native.ZKB_EINVAL
    assert "power of 2" in _native.last_error()
    jobs[1].n = 8
    assert lib.zkb_ntt_batch(ctypes.byref(fr), jobs, 2, None, 0, None, None) == _native.ZKB_EWORKSPACE
    msm = (_native.ZkbMsmJob * 2)()
    msm[0].n, msm[0].result = -1, 64
    assert lib.zkb_msm_batch(msm, 2, None, 0, None) == _native.ZKB_EINVAL
    assert "negative point count" in _native.last_error()
    msm[0].n, msm[0].window_size = 4, 21
    assert lib.zkb_msm_batch_workspace_bytes(msm, 1) == 0
    assert "window_size" in _native.last_error()


def test_gpu_entry_points_reject_bad_arguments_before_touching_the_device():
    lib = _native.lib()
    f = _native.make_field(R)
    assert lib.zkb_field_mul(ctypes.byref(f), 0, 2, 0, 1, 0, 5, None) == _native.ZKB_EINVAL
    assert lib.zkb_ntt(ctypes.byref(f), 8, 16, 6, 0, None, None, None, 0, None) == _native.ZKB_EINVAL
    assert "power of 2" in _native.last_error()
    assert lib.zkb_msm(8, 8, 10, 21, 8, None, 0, None) == _native.ZKB_EINVAL
    assert "window_size" in _native.last_error()
    assert lib.zkb_field_mul(ctypes.byref(f), 0, 1, 0, 1, 0, 0, None) == _native.ZKB_OK  # n = 0 is a no-op
    # misaligned row buffers are refused on the host, before any launch
    assert lib.zkb_field_mul(ctypes.byref(f), 8, 1, 32, 1, 64, 4, None) == _native.ZKB_EINVAL
    assert "16-byte aligned" in _native.last_error()
    assert lib.zkb_msm(64, 64, 4, 0, 4, None, 0, None) == _native.ZKB_EINVAL
    assert "8-byte aligned" in _native.last_error()


# ------------------------------------------------------------------
# Field256: the reference's constructor, constants and validation
# ------------------------------------------------------------------


def test_montgomery_constants_match_published_values():
    assert BN254_FR._n_inv == 0xC2E1F593EFFFFFFF
    assert BN254_FQ._n_inv == 0x87D20782E4866389
    for field in (BN254_FR, BN254_FQ):
        assert field._n_inv * field.modulus % 2**64 == 2**64 - 1
        assert field._r2 == pow(2, 512, field.modulus)


def test_cuda_source_carries_the_modulus_constants():
    source = BN254_FR.cuda_source()
    assert "#define ZK_NINV 0xc2e1f593efffffffULL" in source
    assert "#define ZK_P0 0x43e1f593f0000001ULL" in source
    assert "#define ZK_ONE0 0xac96341c4ffffffbULL" in source
    assert curve_gpu.cuda_source().startswith(BN254_FQ.cuda_source().splitlines()[0])


@pytest.mark.parametrize("modulus", [2, 1, 0, -7, 2**64, 2**255 + 1, 2**256 - 189])
def test_invalid_moduli_raise(modulus):
    with pytest.raises(ValueError, match="odd and in"):
        Field256(modulus)


def test_float_modulus_raises():
    with pytest.raises(TypeError):
        Field256(7.0)


def test_repr_names_the_modulus():
    assert repr(Field256(3)) == "Field256(0x3)"


@pytest.mark.parametrize(
    "bad",
    [np.zeros((3, 4), dtype=np.int64), np.zeros((3, 3), dtype=np.uint64), np.zeros(12, dtype=np.uint64), [[0, 0, 0, 0]]],
    ids=["int64", "3-limbs", "flat", "list"],
)
def test_malformed_rows_raise(bad):
    with pytest.raises(TypeError, match=r"\(n, 4\) uint64"):
        BN254_FR.mul(bad, np.zeros((1, 4), dtype=np.uint64))


def test_mismatched_row_counts_raise():
    with pytest.raises(ValueError, match="broadcast"):
        BN254_FR.mul(np.zeros((2, 4), dtype=np.uint64), np.zeros((3, 4), dtype=np.uint64))


@pytest.mark.parametrize(
    ("field", "n", "message"),
    [(BN254_FR, 6, "power of 2"), (BN254_FQ, 4, "not divisible"), (Field256(2**255 - 1), 2, "odd prime")],
    ids=["size-6", "fq-size-4", "composite"],
)
def test_ntt_rejects_unsupported_sizes(field, n, message):
    with pytest.raises(ValueError, match=message):
        field.ntt(np.zeros((n, 4), dtype=np.uint64))


def test_ntt_beyond_two_adicity_raises():
    with pytest.raises(ValueError, match="not supported"):
        roots.get_ntt_root(2**29, R)


def test_curve_shape_checks():
    with pytest.raises(TypeError, match=r"\(n, 3, 4\) uint64 array of Jacobian points"):
        curve_gpu.add(np.zeros((1, 2, 4), dtype=np.uint64), np.zeros((1, 2, 4), dtype=np.uint64))
    with pytest.raises(TypeError, match=r"\(n, 2, 4\) uint64 array of affine points"):
        curve_gpu.add_affine(np.zeros((1, 3, 4), dtype=np.uint64), np.zeros((1, 3, 4), dtype=np.uint64))
    with pytest.raises(ValueError, match="broadcast"):
        curve_gpu.add(np.zeros((2, 3, 4), dtype=np.uint64), np.zeros((3, 3, 4), dtype=np.uint64))
    with pytest.raises(ValueError, match="triples"):
        curve_gpu.jacobian_to_device([(1, 2)])
    with pytest.raises(ValueError, match="point at infinity"):
        curve_gpu.affine_to_device([G, Point.identity()])


# ------------------------------------------------------------------
# MSM argument validation (reference tests/test_msm.py:355-369)
# ------------------------------------------------------------------


def test_msm_validates_arguments():
    with pytest.raises(ValueError, match="Length mismatch"):
        msm_gpu.msm_pippenger_gpu([G.x], [G.y], [1, 2])
    for bad_window in (0, 17):
        with pytest.raises(ValueError, match="window_size"):
            msm_gpu.msm_pippenger_gpu([G.x], [G.y], [1], window_size=bad_window)
    with pytest.raises(TypeError, match="scalars must contain integers"):
        msm_gpu.msm_pippenger_gpu([G.x], [G.y], [1.5])
    with pytest.raises(TypeError):
        msm_gpu.msm_pippenger_gpu([G.x], [G.y], [1], P)
    assert msm_gpu.msm_pippenger_gpu([], [], []) == Point.identity()


def test_window_size_cost_model_is_the_references():
    assert [msm_gpu.pippenger_window_size(n) for n in (0, 100, 1_000, 10_000, 100_000)] == [1, 5, 7, 10, 13]


# ------------------------------------------------------------------
# Points and roots
# ------------------------------------------------------------------


def test_point_validation_and_value_semantics():
    assert G.is_on_curve() and Point(1, P - 2) == -G
    assert -Point.identity() == Point.identity()
    with pytest.raises(ValueError, match="not on the BN254 curve"):
        Point(1, 3)
    with pytest.raises(ValueError):
        Point(1, None)
    assert Point(1 + P, 2 - P) == G and hash(Point(1 + P, 2)) == hash(G)
    with pytest.raises(ValueError, match="no affine coordinates"):
        Point.identity().affine()


def test_roots_of_unity():
    k = golden("known.json")
    assert roots.get_ntt_root(2**28, R) == h(k["root_2_28"])
    assert roots.get_ntt_root(2**28, R, non_residue=7) == h(k["root_2_28_generator_7"])
    assert roots.quadratic_non_residue(R) == 5
    assert roots.default_coset_offset(8, R) == 5
    for kk in (1, 2, 10, 20, 27):
        assert roots.get_ntt_root(2**kk, R) == pow(h(k["root_2_28"]), 2 ** (28 - kk), R)
    with pytest.raises(ValueError, match="odd prime"):
        roots.get_ntt_root(2, 2**255 - 1)


# ------------------------------------------------------------------
# No CPU fallback
# ------------------------------------------------------------------


def test_device_operations_fail_loudly_without_a_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA device"):
        BN254_FR.from_ints([1, 2, 3])
    with pytest.raises(RuntimeError, match="CUDA device"):
        msm_gpu.msm_pippenger_gpu([G.x], [G.y], [5])
    with pytest.raises(RuntimeError, match="CUDA device"):
        curve_gpu.double(np.zeros((1, 3, 4), dtype=np.uint64))


def test_product_never_imports_the_oracle():
    pkg = ROOT / "zk-gpu-accelerator_b200" / "zkgpu"
    for src in pkg.glob("*.py"):
        text = src.read_text()
        assert "import oracle" not in text and "from oracle" not in text, src.name


# ------------------------------------------------------------------
# Per-size tuning tables and the autotuner's cache (no GPU needed)
# ------------------------------------------------------------------


def test_per_size_tables_drive_the_plans(tmp_path):
    from zkgpu import autotune

    lib = _native.lib()
    with pytest.raises(ValueError, match="unknown per-size"):
        _native.tune_set_sized("msm.bogus", 10, 3)
    with pytest.raises(ValueError, match="1..20"):
        _native.tune_set_sized("msm.window", 10, 21)
    with pytest.raises(ValueError, match="0..32"):
        _native.tune_set_sized("msm.window", 40, 3)
    model = lib.zkb_msm_default_window(3000)
    try:
        _native.tune_set_sized("msm.window", 12, 7)  # 3000 points round up to 2^12
        assert lib.zkb_msm_default_window(3000) == 7
        assert lib.zkb_msm_default_window(5000) == lib.zkb_msm_default_window(8192)  # the 2^13 entry: none
        _native.tune_set_sized("ntt.max_log_radix", 9, 8)  # 2^9 rows in two passes
        assert lib.zkb_ntt_workspace_bytes(512) == 512 * 32
        assert lib.zkb_ntt_workspace_bytes(256) == 0
        table = {"device": "test-gpu", "msm": {12: {"window": 9}},
                 "ntt": {20: {"max_log_radix": 10, "cta_log_elems": 11, "threads": 256}}}
        path = autotune.save(table, tmp_path / "tune.json")
        back = autotune.load(path, key="test-gpu")
        assert back["msm"]["12"]["window"] == 9 and back["ntt"]["20"]["threads"] == 256
        assert autotune.load(path, key="other-gpu") is None
        autotune.apply(back)
        assert _native.tune_get_sized("msm.window", 12) == 9
        assert _native.tune_get_sized("ntt.cta_log_elems", 20) == 11
    finally:
        autotune.clear()
    assert lib.zkb_msm_default_window(3000) == model
    assert lib.zkb_ntt_workspace_bytes(512) == 0


# ------------------------------------------------------------------
# Fixed-base tables: host-side checks (no GPU needed)
# ------------------------------------------------------------------


def test_fixed_base_table_window_is_checked_first():
    from zkgpu.msm_gpu import FixedBaseTable

    for w in (7, 25, 0):
        with pytest.raises(ValueError, match="window_size must be in 8..24"):
            FixedBaseTable(np.zeros((4, 2, 4), dtype=np.uint64), w)
    with pytest.raises(TypeError):
        FixedBaseTable(np.zeros((4, 2, 4), dtype=np.uint64), 16.0)


def test_table_job_rows_and_their_limit():
    """msm_table_jobs puts the table in place of the base set's prefix, with its window."""
    import types

    import torch

    from zkgpu.prover import msm_table_jobs

    table = types.SimpleNamespace(n=100, window_size=16, table=torch.zeros(8, dtype=torch.uint64))
    jobs = msm_table_jobs(table, [(111, 222, 100, 333), (111, 444, 5, 555)])
    assert [(j.points, j.scalars, j.n, j.result, j.window_size) for j in jobs] == [
        (table.table.data_ptr(), 222, 100, 333, 16), (table.table.data_ptr(), 444, 5, 555, 16)]
    with pytest.raises(ValueError, match="101 points over a table of 100"):
        msm_table_jobs(table, [(111, 222, 101, 333)])


def test_table_sizes_follow_the_window():
    from zkgpu import _native

    lib = _native.lib()
    assert lib.zkb_msm_table_bytes(1 << 20, 16) == (1 << 20) * 16 * 64
    assert lib.zkb_msm_table_bytes(1000, 22) == 1000 * 12 * 64
    assert lib.zkb_msm_table_bytes(1000, 7) == 0 and lib.zkb_msm_table_bytes(1000, 25) == 0
    assert lib.zkb_msm_table_bytes(0, 16) == 0
