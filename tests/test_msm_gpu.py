"""
zkgpu.msm_gpu on the GPU: the affine result bit-exact against the
reference's Pippenger on the same inputs (golden fixtures: its test cases and
seeded 2^12 / 2^14 / 2^16 instances), every window size, skewed scalars, and
at the config sizes (2^22 points) through size-independent identities and a
2^16 subset against the C oracle.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from conftest import golden, hs
from oracle import c_oracle as co
from oracle import pyoracle as po
from zkgpu import _native, curve_gpu, msm_gpu
from zkgpu import workloads as wl
from zkgpu.curve import G, P, Point, R
from zkgpu.msm_gpu import msm_pippenger_gpu, msm_pippenger_rows

pytestmark = pytest.mark.gpu


def expected_point(case) -> Point:
    return Point.identity() if case["expected"] is None else Point(*hs(case["expected"]))


def run_case(case, window_size=None) -> Point:
    pts = [hs(p) for p in case["points"]]
    sc = [int(s) for s in case["raw_scalars"]] if "raw_scalars" in case else hs(case["scalars"])
    return msm_pippenger_gpu(
        np.array([p[0] for p in pts], dtype=object),
        np.array([p[1] for p in pts], dtype=object),
        np.array(sc, dtype=object),
        window_size=window_size,
    )


@pytest.mark.parametrize("window_size", [None, 1, 2, 3, 5, 8, 11, 13, 16])
@pytest.mark.parametrize("case", golden("msm.json")["cases"], ids=lambda c: c["name"])
def test_msm_matches_the_references(case, window_size):
    assert run_case(case, window_size) == expected_point(case)


def _bases(n: int, seed: int):
    return curve_gpu.mul_generator(wl.base_scalars(seed, n))


@pytest.mark.parametrize("case", golden("msm.json")["seeded"], ids=lambda c: f"{c['kind']}-{c['n']}")
def test_seeded_msm_matches_the_references(case):
    n = case["n"]
    bases = _bases(n, case["base_seed"])
    gen = wl.uniform_fr if case["kind"] == "uniform" else wl.skewed_scalars
    sc = gen(case["scalar_seed"], n)
    for w in (None, 4, 9, 12, 16):
        assert msm_pippenger_rows(bases, sc, window_size=w) == expected_point(case), w


def _msm_raw(points, scalars, n, w):
    """zkb_msm through the C ABI directly, for window sizes above the API's 16."""
    import torch

    lib = _native.lib()
    ws_bytes = lib.zkb_msm_workspace_bytes(n, w)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    out = torch.empty(9, dtype=torch.int64, device="cuda")
    _native.check(lib.zkb_msm(points.data_ptr(), scalars.data_ptr(), n, w, out.data_ptr(), ws.data_ptr(),
                              ws_bytes, _native.stream_ptr()))
    return msm_gpu._result_point(out.cpu().numpy().view(np.uint64))


@pytest.mark.parametrize("w", [17, 18, 20])
def test_internal_windows_beyond_16(w):
    case = golden("msm.json")["seeded"][0]
    n = case["n"]
    import torch

    bases = _bases(n, case["base_seed"])
    gen = wl.uniform_fr if case["kind"] == "uniform" else wl.skewed_scalars
    sc = torch.from_numpy(gen(case["scalar_seed"], n)).cuda()
    assert _msm_raw(bases, sc, n, w) == expected_point(case)


def test_bucket_edge_cases():
    assert msm_pippenger_gpu([G.x, G.x], [G.y, P - G.y], [7, 7]) == Point.identity()
    assert msm_pippenger_gpu([G.x, G.x], [G.y, G.y], [5, 5]) == Point(*po.scalar_mul(po.G, 10))
    assert msm_pippenger_gpu([G.x, G.x], [G.y, G.y], [0, 0]) == Point.identity()


def test_reduces_scalars_mod_r():
    three = po.scalar_mul(po.G, 3)
    for scalar in (-5, R, R + 7, 2**300 + 1):
        want = po.scalar_mul(three, scalar % R)
        assert msm_pippenger_gpu([three[0]], [three[1]], [scalar]) == (Point.identity() if want is None else Point(*want))


def test_returns_a_point():
    assert msm_pippenger_gpu([], [], []) == Point.identity()
    result = msm_pippenger_gpu([G.x], [G.y], [R])
    assert isinstance(result, Point) and result.is_identity()
    assert msm_pippenger_gpu([G.x, G.x], [G.y, G.y], [2, 3]) == Point(*po.scalar_mul(po.G, 5))


def test_off_curve_points_are_rejected_on_the_device():
    with pytest.raises(ValueError, match=r"\(1, 3\) is not on the BN254 curve"):
        msm_pippenger_gpu([1], [3], [5])
    with pytest.raises(ValueError, match="not on the BN254 curve"):
        msm_pippenger_gpu([G.x, 1, G.x], [G.y, 3, G.y], [1, 2, 3])


def test_heavy_bucket_and_boolean_scalars():
    pts = [po.scalar_mul(po.G, k) for k in range(1, 301)]
    xs, ys = [p[0] for p in pts], [p[1] for p in pts]
    scalar = 2**200 + 12345
    assert msm_pippenger_gpu(xs, ys, [scalar] * 300) == Point(*po.scalar_mul(po.G, sum(range(1, 301)) * scalar % R))
    bools = [k % 3 != 0 for k in range(300)]
    want = po.msm_double_and_add(pts, [int(b) for b in bools])
    assert msm_pippenger_gpu(xs, ys, [int(b) for b in bools], window_size=9) == Point(*want)


@pytest.mark.parametrize("case", golden("msm.json")["seeded"][:2], ids=lambda c: f"{c['kind']}-{c['n']}")
def test_inlined_products_give_the_same_point(case):
    """The bucket, merge, reduction and finalize kernels compiled with every product expanded
    in place (msm.call_products = 0) give the reference's point as the default shared-product
    kernels do."""
    n = case["n"]
    bases = _bases(n, case["base_seed"])
    gen = wl.uniform_fr if case["kind"] == "uniform" else wl.skewed_scalars
    sc = gen(case["scalar_seed"], n)
    try:
        _native.tune_set("msm.call_products", 0)
        for w in (None, 7):
            assert msm_pippenger_rows(bases, sc, window_size=w) == expected_point(case), w
    finally:
        _native.tune_set("msm.call_products", 1)


@pytest.mark.parametrize("sort", [0, 1], ids=["radix-sort", "counting-sort"])
def test_both_pair_sorts_give_the_references_points(sort):
    """The radix sort of all pairs (msm.sort = 0) and the counting sort that skips zero digits
    (msm.sort = 1, the default) give the reference's points: the seeded uniform and skewed cases,
    the bucket edge cases, a heavy bucket, boolean and all-zero scalars, and a batch."""
    from zkgpu import batch

    try:
        _native.tune_set("msm.sort", sort)
        for case in golden("msm.json")["seeded"][:2]:
            n = case["n"]
            bases = _bases(n, case["base_seed"])
            gen = wl.uniform_fr if case["kind"] == "uniform" else wl.skewed_scalars
            sc = gen(case["scalar_seed"], n)
            for w in (None, 5, 16):
                assert msm_pippenger_rows(bases, sc, window_size=w) == expected_point(case), (case["kind"], w)
        test_bucket_edge_cases()
        test_heavy_bucket_and_boolean_scalars()
        pts = [po.scalar_mul(po.G, k) for k in range(1, 65)]
        assert msm_pippenger_gpu([p[0] for p in pts], [p[1] for p in pts], [0] * 64) == Point.identity()
        case = golden("msm.json")["seeded"][0]
        bases = _bases(case["n"], case["base_seed"])
        import torch

        sc = torch.from_numpy(wl.uniform_fr(case["scalar_seed"], case["n"])).cuda()
        zeros = torch.zeros_like(sc)
        got = batch.msm_batch([bases, bases[:100], bases], [sc, sc[:100], zeros])
        assert got[0] == expected_point(case) and got[2] == Point.identity()
        assert got[1] == msm_pippenger_rows(bases[:100], sc[:100])
    finally:
        _native.tune_set("msm.sort", 1)


def test_self_test_passes():
    msm_gpu.compile_kernels()


# ------------------------------------------------------------------
# Config sizes: 2^22 points (config 3), uniform and skewed scalars
# ------------------------------------------------------------------


@pytest.fixture(scope="module")
def big_bases():
    return _bases(1 << 22, 3)


def test_2_22_subset_matches_c_oracle(big_bases):
    """Config 3's subset check: the first 2^16 of the 2^22 inputs against the C oracle."""
    m = 1 << 16
    for sc in (wl.uniform_fr(3, 1 << 22)[:m], wl.skewed_scalars(4, 1 << 22)[:m]):
        got = msm_pippenger_rows(big_bases[:m], sc)
        out = co.msm(big_bases[:m].cpu().numpy(), sc, 16, threads=os.cpu_count() or 1)
        want = Point.identity() if out[8] else Point(*wl.rows_to_ints(out[:8].reshape(2, 4)))
        assert got == want


@pytest.mark.parametrize("kind", ["uniform", "skewed"])
def test_2_22_linearity_and_split(big_bases, kind):
    """sum s_i P_i + sum t_i P_i == sum (s_i + t_i) P_i, and the sum of two halves is the whole."""
    n = 1 << 22
    gen = wl.uniform_fr if kind == "uniform" else wl.skewed_scalars
    s, t = gen(3, n), gen(4, n)
    whole_s = msm_pippenger_rows(big_bases, s)
    whole_t = msm_pippenger_rows(big_bases, t)
    st = np.array(wl.rows_to_ints(s), dtype=object) + np.array(wl.rows_to_ints(t), dtype=object)
    st_rows = np.array([[(v % R >> (64 * j)) & (2**64 - 1) for j in range(4)] for v in st], dtype=np.uint64)
    assert whole_s + whole_t == msm_pippenger_rows(big_bases, st_rows)
    h = n // 2 + 12345
    assert msm_pippenger_rows(big_bases[:h], s[:h]) + msm_pippenger_rows(big_bases[h:], s[h:]) == whole_s
    assert not whole_s.is_identity()


def test_workspace_too_small_is_an_error():
    import torch

    lib = _native.lib()
    bases = _bases(64, 9)
    sc = torch.from_numpy(wl.uniform_fr(9, 64)).cuda()
    out = torch.empty(9, dtype=torch.int64, device="cuda")
    status = lib.zkb_msm(bases.data_ptr(), sc.data_ptr(), 64, 8, out.data_ptr(), None, 0, _native.stream_ptr())
    assert status == _native.ZKB_EWORKSPACE
    assert "workspace" in _native.last_error()
    assert ctypes.c_int(status).value == 5


# ------------------------------------------------------------------
# Affine rounds (batch-affine bucket additions before the XYZZ levels)
# ------------------------------------------------------------------


def _with_knobs(knobs: dict, fn):
    old = {k: _native.tune_get(k) for k in knobs}
    try:
        for k, v in knobs.items():
            _native.tune_set(k, v)
        return fn()
    finally:
        for k, v in old.items():
            _native.tune_set(k, v)


@pytest.mark.parametrize("rounds", [1, 2, 3, 6])
@pytest.mark.parametrize("batch", [8, 64])
@pytest.mark.parametrize("case", golden("msm.json")["seeded"], ids=lambda c: f"{c['kind']}-{c['n']}")
def test_affine_rounds_give_the_references_points(case, rounds, batch):
    """Forced affine rounds (each bucket list halved by affine additions with one inversion per
    block) at the seeded sizes, uniform and skewed, against the reference's points."""
    n = case["n"]
    bases = _bases(n, case["base_seed"])
    gen = wl.uniform_fr if case["kind"] == "uniform" else wl.skewed_scalars
    sc = gen(case["scalar_seed"], n)
    knobs = {"msm.affine_rounds": rounds, "msm.affine_batch": batch}
    for w in (None, 6, 13):
        assert _with_knobs(knobs, lambda: msm_pippenger_rows(bases, sc, window_size=w)) == expected_point(case), w


@pytest.mark.parametrize("rounds", [1, 2, 4])
def test_affine_rounds_special_cases(rounds):
    """Buckets whose pairs hit every case of the affine addition: P + P (a doubling),
    P + (-P) (infinity, which later rounds and the XYZZ levels must skip), infinity + Q and
    Q + infinity (copies), and odd list lengths; against double-and-add on the CPU."""
    k = [1, 2, 3, 5, 8]
    base = [po.scalar_mul(po.G, v) for v in k]
    neg = [(x, (P - y) % P) for x, y in base]
    pts = []
    for i in range(40):  # runs of equal points, their negatives, and mixtures
        pts += [base[i % 5]] * (1 + i % 3) + [neg[i % 5]] * (i % 2) + [base[(i + 1) % 5]]
    scalars_list = [[1] * len(pts), [2**64 + 3] * len(pts), [(i % 7) + 1 for i in range(len(pts))]]
    xs, ys = [p[0] for p in pts], [p[1] for p in pts]
    for scalars in scalars_list:
        want = po.msm_double_and_add(pts, scalars)
        want = Point.identity() if want is None else Point(*want)
        got = _with_knobs({"msm.affine_rounds": rounds, "msm.affine_batch": 8},
                          lambda: msm_pippenger_gpu(xs, ys, scalars, window_size=4))
        assert got == want
    # a bucket that sums to exactly infinity: P, -P, 2P, -2P, all with one scalar
    two = po.scalar_mul(po.G, 2)
    cancel = [base[0], neg[0], two, (two[0], (P - two[1]) % P)]
    got = _with_knobs({"msm.affine_rounds": rounds, "msm.affine_batch": 8},
                      lambda: msm_pippenger_gpu([p[0] for p in cancel], [p[1] for p in cancel], [9] * 4))
    assert got == Point.identity()


def test_affine_rounds_in_batches_and_fixed_base_tables():
    """Batched MSMs (one pipeline for several jobs) and MSMs over a fixed-base table with
    forced affine rounds give the points of the plain path."""
    from zkgpu import batch
    from zkgpu.msm_gpu import FixedBaseTable

    n = 1 << 14
    bases = _bases(n, 77)
    scs = [wl.uniform_fr(78, n), wl.skewed_scalars(79, n // 2), wl.uniform_fr(80, 1000)]
    pts = [bases, bases[: n // 2], bases[:1000]]
    want = [msm_pippenger_rows(p, s) for p, s in zip(pts, scs)]
    knobs = {"msm.affine_rounds": 3, "msm.affine_batch": 16}
    assert _with_knobs(knobs, lambda: batch.msm_batch(pts, scs)) == want
    table = FixedBaseTable(bases, 12)
    got = _with_knobs(knobs, lambda: batch.msm_fixed_batch(table, scs[:2]))
    assert got == want[:2]


def test_affine_rounds_with_inlined_products():
    case = golden("msm.json")["seeded"][0]
    n = case["n"]
    bases = _bases(n, case["base_seed"])
    gen = wl.uniform_fr if case["kind"] == "uniform" else wl.skewed_scalars
    sc = gen(case["scalar_seed"], n)
    knobs = {"msm.affine_rounds": 2, "msm.affine_batch": 32, "msm.call_products": 0}
    assert _with_knobs(knobs, lambda: msm_pippenger_rows(bases, sc)) == expected_point(case)


# ------------------------------------------------------------------
# Bucket reduction by warps ("msm.reduce_log_segment": buckets a lane sums at level 1)
# ------------------------------------------------------------------


@pytest.mark.parametrize("log_l", [0, 1, 2, 3, 4, 5, 8])
@pytest.mark.parametrize("case", golden("msm.json")["seeded"], ids=lambda c: f"{c['kind']}-{c['n']}")
def test_every_reduction_segment_gives_the_references_points(case, log_l):
    """Every segment length of the first reduction level (1..256 buckets a lane), at windows
    whose buckets take one level (w <= 5 at 16 a lane), two, and three (w = 20: 2^19
    buckets, 1,024 chunks at level 2), against the reference's points."""
    import torch

    n = case["n"]
    bases = _bases(n, case["base_seed"])
    gen = wl.uniform_fr if case["kind"] == "uniform" else wl.skewed_scalars
    sc = gen(case["scalar_seed"], n)
    sc_dev = torch.from_numpy(sc).cuda()
    knobs = {"msm.reduce_log_segment": log_l}
    for w in (None, 1, 5, 11, 16):
        assert _with_knobs(knobs, lambda: msm_pippenger_rows(bases, sc, window_size=w)) == expected_point(case), w
    assert _with_knobs(knobs, lambda: _msm_raw(bases, sc_dev, n, 20)) == expected_point(case)


def test_reduction_segments_in_batches_and_fixed_base_tables():
    """The batch and fixed-base forms (one bucket set per job) at segment lengths 1, 16, 256,
    against each job alone at the default knobs."""
    from zkgpu import batch

    n = 3000
    bases = _bases(n, 71)
    scs = [wl.uniform_fr(72, n), wl.skewed_scalars(73, 1777), wl.uniform_fr(74, 5)]
    alone = [msm_pippenger_rows(bases[: s.shape[0]], s) for s in scs]
    table = msm_gpu.FixedBaseTable(bases, 12)
    for log_l in (0, 4, 8):
        knobs = {"msm.reduce_log_segment": log_l}
        got = _with_knobs(knobs, lambda: batch.msm_batch([bases[: s.shape[0]] for s in scs], scs))
        assert got == alone, log_l
        got_t = _with_knobs(knobs, lambda: batch.msm_fixed_batch(table, scs))
        assert got_t == alone, log_l
