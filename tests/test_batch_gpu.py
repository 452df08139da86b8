"""
Batched forms on the GPU (zkgpu.batch): every job of an NTT batch (one
persistent launch) and of an MSM batch (jobs grouped by window size, groups on
side streams) gives exactly the rows / point of the one-at-a-time call, which
the other test files pin to the reference; a sample is also checked against
the C oracle directly. CUDA-graph replay of a captured BatchPlan gives the
same results as eager runs, also after new inputs are copied in.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import c_oracle as co
from zkgpu import _native, batch, curve_gpu
from zkgpu import workloads as wl
from zkgpu.curve import Point
from zkgpu.field256_gpu import BN254_FR
from zkgpu.msm_gpu import msm_pippenger_rows

pytestmark = pytest.mark.gpu


def _rows_fr(seed: int, n: int):
    return BN254_FR.to_montgomery(wl.uniform_fr(seed, n))


# ------------------------------------------------------------------
# NTT batches
# ------------------------------------------------------------------

MIXED_SIZES = [1, 2, 8, 1 << 10, 1 << 12, 1 << 13, 1 << 9, 1 << 16, 1 << 20, 4, 1 << 11, 1 << 18]


def test_ntt_batch_matches_single_transforms():
    xs = [_rows_fr(100 + k, n) for k, n in enumerate(MIXED_SIZES)]
    inv = [k % 2 == 1 for k in range(len(xs))]
    cos = [5 if k % 3 == 0 else None for k in range(len(xs))]
    outs = batch.ntt_batch(xs, invert=inv, coset=cos)
    for x, y, i, c in zip(xs, outs, inv, cos, strict=True):
        assert bool((y == BN254_FR.ntt(x, invert=i, coset=c)).all()), (int(x.shape[0]), i, c)


def test_ntt_batch_of_64_log_uniform_sizes_matches_c_oracle():
    """Config 4's NTT half: 64 transforms with sizes log-uniform in 2^10..2^20."""
    rng = np.random.default_rng(6)
    sizes = [1 << int(v) for v in rng.integers(10, 21, size=64)]
    xs = [_rows_fr(200 + k, n) for k, n in enumerate(sizes)]
    outs = batch.ntt_batch(xs)
    threads = os.cpu_count() or 1
    for k, (x, y) in enumerate(zip(xs, outs, strict=True)):
        if k % 8 == 0:  # a sample against the oracle, every job against the single call
            want = co.ntt(x.cpu().numpy(), threads=threads)
            assert np.array_equal(y.cpu().numpy(), want), sizes[k]
        assert bool((y == BN254_FR.ntt(x)).all()), sizes[k]


def test_ntt_batch_with_three_pass_transforms():
    """At most 8 bits per pass: 2^17..2^20 take three passes, whose tiles wait on two earlier passes."""
    try:
        _native.tune_set("ntt.max_log_radix", 8)
        xs = [_rows_fr(300 + k, n) for k, n in enumerate([1 << 20, 1 << 17, 1 << 12, 1 << 18, 64])]
        outs = batch.ntt_batch(xs, invert=[False, True, False, True, False], coset=[5, None, 7, 5, None])
        for x, y, i, c in zip(xs, outs, [False, True, False, True, False], [5, None, 7, 5, None], strict=True):
            assert bool((y == BN254_FR.ntt(x, invert=i, coset=c)).all()), int(x.shape[0])
    finally:
        _native.tune_set("ntt.max_log_radix", 0)


def test_ntt_batch_round_trip_and_limits():
    xs = [_rows_fr(400 + k, 1 << k) for k in range(2, 15)]
    back = batch.ntt_batch(batch.ntt_batch(xs, coset=5), invert=True, coset=5)
    for x, b in zip(xs, back, strict=True):
        assert bool((x == b).all())
    assert batch.ntt_batch([]) == []
    with pytest.raises(ValueError, match="at most 64"):
        batch.ntt_batch([xs[0]] * 65)
    with pytest.raises(ValueError, match="power of 2"):
        batch.ntt_batch([_rows_fr(1, 6)])


# ------------------------------------------------------------------
# MSM batches
# ------------------------------------------------------------------


@pytest.fixture(scope="module")
def base_set():
    return curve_gpu.mul_generator(wl.base_scalars(6, 1 << 16))


def test_msm_batch_matches_single_msms(base_set):
    sizes = [0, 1, 2, 100, 1 << 12, 1 << 16, 3000, 1 << 14, 1 << 12]
    windows = [None, None, 3, None, 16, None, 7, 12, 16]
    pts = [base_set[:n] for n in sizes]
    scs = [wl.uniform_fr(500 + k, n) if k % 2 else wl.skewed_scalars(500 + k, n) for k, n in enumerate(sizes)]
    got = batch.msm_batch(pts, scs, window_sizes=windows)
    for k, (p, s, w) in enumerate(zip(pts, scs, windows, strict=True)):
        assert got[k] == msm_pippenger_rows(p, s, window_size=w, check_points=False), (sizes[k], w)
    assert got[0] == Point.identity()


def test_msm_batch_of_32_log_uniform_sizes_matches_c_oracle(base_set):
    """Config 4's MSM half (over a 2^16 base set here): 32 MSMs with log-uniform sizes over
    prefixes of one resident base set; default windows, so several window groups run at once."""
    rng = np.random.default_rng(6)
    sizes = [int(2 ** v) for v in rng.uniform(12, 16, size=32)]
    pts = [base_set[:n] for n in sizes]
    scs = [wl.uniform_fr(600 + k, n) for k, n in enumerate(sizes)]
    got = batch.msm_batch(pts, scs)
    host = base_set.cpu().numpy()
    for k in range(0, 32, 4):
        n = sizes[k]
        w = int(_native.lib().zkb_msm_default_window(n))
        out = co.msm(host[:n], scs[k], w, threads=os.cpu_count() or 1)
        want = Point.identity() if out[8] else Point(*wl.rows_to_ints(out[:8].reshape(2, 4)))
        assert got[k] == want, n
    for k in range(1, 32, 4):
        assert got[k] == msm_pippenger_rows(pts[k], scs[k], check_points=False), sizes[k]


def test_msm_batch_argument_errors(base_set):
    with pytest.raises(ValueError, match="Length mismatch"):
        batch.msm_batch([base_set[:4]], [])
    with pytest.raises(ValueError, match="window_size"):
        batch.msm_batch([base_set[:4]], [wl.uniform_fr(1, 4)], window_sizes=[21])
    assert batch.msm_batch([], []) == []


# ------------------------------------------------------------------
# CUDA-graph replay
# ------------------------------------------------------------------


def test_captured_batch_plan_replays_exactly(base_set):
    import torch

    ntt_in = [_rows_fr(700 + k, n).clone() for k, n in enumerate([1 << 12, 1 << 16, 1 << 10])]
    msm_sc = [torch.from_numpy(wl.uniform_fr(710 + k, n)).cuda() for k, n in enumerate([1 << 12, 5000])]
    plan = batch.BatchPlan(
        ntt_jobs=[(ntt_in[0], False, None), (ntt_in[1], True, 5), (ntt_in[2], False, 5)],
        msm_jobs=[(base_set[: 1 << 12], msm_sc[0], None), (base_set[:5000], msm_sc[1], 9)],
    )
    plan.run()
    eager_ntt = [y.clone() for y in plan.ntt_outputs]
    eager_msm = plan.msm_points_out()
    plan.capture()
    plan.replay()
    plan.check_status()
    assert all(bool((a == b).all()) for a, b in zip(eager_ntt, plan.ntt_outputs, strict=True))
    assert plan.msm_points_out() == eager_msm
    # new data of the same shapes: copy into the bound inputs, replay, compare with fresh calls
    ntt_in[1].copy_(_rows_fr(720, 1 << 16))
    msm_sc[0].copy_(torch.from_numpy(wl.uniform_fr(721, 1 << 12)))
    plan.replay()
    assert bool((plan.ntt_outputs[1] == BN254_FR.ntt(ntt_in[1], invert=True, coset=5)).all())
    assert plan.msm_points_out()[0] == msm_pippenger_rows(base_set[: 1 << 12], msm_sc[0], check_points=False)
    assert plan.launches_per_run > 0


def test_concurrent_plan_equals_the_sequential_plan_and_replays(base_set):
    """MSM batch on a high-priority stream, transforms on a low-priority one: same rows and
    points as the plain order, eagerly and from a captured graph."""
    import torch

    x = _rows_fr(800, 1 << 16)
    sc = [torch.from_numpy(wl.uniform_fr(801, 1 << 15)).cuda(), torch.from_numpy(wl.skewed_scalars(802, 1 << 16)).cuda()]
    jobs = dict(ntt_jobs=[(x, False, None), (x, True, 5)],
                msm_jobs=[(base_set[: 1 << 15], sc[0], None), (base_set, sc[1], None)])
    seq = batch.BatchPlan(**jobs)
    seq.run()
    conc = batch.BatchPlan(**jobs, concurrent=True)
    conc.run()
    torch.cuda.synchronize()
    assert all(bool((a == b).all()) for a, b in zip(seq.ntt_outputs, conc.ntt_outputs, strict=True))
    assert seq.msm_points_out() == conc.msm_points_out()
    conc.capture()
    for y in conc.ntt_outputs:
        y.zero_()
    conc.msm_results.zero_()
    conc.replay()
    torch.cuda.synchronize()
    assert all(bool((a == b).all()) for a, b in zip(seq.ntt_outputs, conc.ntt_outputs, strict=True))
    assert seq.msm_points_out() == conc.msm_points_out()


# ------------------------------------------------------------------
# The persistent launch's bounded dependency wait
# ------------------------------------------------------------------


def test_ntt_batch_wait_that_runs_out_reports_timeout_then_next_batch_is_exact():
    """A tile of a transform's second pass waits for every tile of its first pass. With the
    wait bounded to one poll ("ntt.batch_spin_limit" = 1), the first second-pass tile of a
    2^22-row transform gives up while the last wave of first-pass tiles is still running: the
    kernel returns, the status word reads ZKB_ETIMEOUT, and the host raises. The default bound
    then gives the exact transform again (the counters and status are reset per launch)."""
    import torch

    x = _rows_fr(171, 1 << 22)
    want = BN254_FR.ntt(x)
    _native.tune_set("ntt.batch_spin_limit", 1)
    try:
        plan = batch.BatchPlan(ntt_jobs=[(x, False, None)])
        plan.run()
        torch.cuda.synchronize()
        assert int(plan.status.item()) == _native.ZKB_ETIMEOUT
        with pytest.raises(RuntimeError):
            plan.check_status()
    finally:
        _native.tune_set("ntt.batch_spin_limit", 0)
    assert _native.tune_get("ntt.batch_spin_limit") == 0
    plan.run()
    plan.check_status()
    assert bool((plan.ntt_outputs[0] == want).all())
    fresh = batch.ntt_batch([x])  # the functional form checks the status itself
    assert bool((fresh[0] == want).all())


def test_batch_plan_over_a_fixed_base_table_matches_the_plain_batch():
    """BatchPlan(table=...) runs the MSM jobs over a fixed-base table of the resident base set
    they are prefixes of; points and rows equal the plain batch's, eager and replayed."""
    from zkgpu.msm_gpu import FixedBaseTable

    n = 1 << 14
    bases = curve_gpu.mul_generator(wl.base_scalars(91, n))
    sizes = [n, 3000, 777, 1 << 12]
    scs = [wl.uniform_fr(92 + k, m) for k, m in enumerate(sizes)]
    import torch

    scs = [torch.from_numpy(s).cuda() for s in scs]
    xs = [_rows_fr(95, 1 << 12), _rows_fr(96, 1 << 9)]
    ref = batch.BatchPlan(ntt_jobs=[(x, False, None) for x in xs], msm_jobs=[(bases[:m], s, None) for m, s in zip(sizes, scs)])
    ref.run()
    for w in (12, 16):
        table = FixedBaseTable(bases, w)
        plan = batch.BatchPlan(ntt_jobs=[(x, False, None) for x in xs],
                               msm_jobs=[(bases[:m], s, None) for m, s in zip(sizes, scs)], table=table)
        plan.run()
        assert bool((plan.msm_results[:4, :9] == ref.msm_results[:4, :9]).all()), w
        assert all(bool((a == b).all()) for a, b in zip(plan.ntt_outputs, ref.ntt_outputs))
        plan.capture()
        plan.replay()
        plan.check_status()
        assert bool((plan.msm_results[:4, :9] == ref.msm_results[:4, :9]).all()), w
    with pytest.raises(ValueError, match="table of"):
        batch.BatchPlan(msm_jobs=[(bases, scs[0], None)], table=FixedBaseTable(bases[:100], 12))
