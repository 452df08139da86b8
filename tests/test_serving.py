"""
The serving scheduler's policy without a GPU (zkgpu.serving.Scheduler):
first-come first-served admission under the HBM budget, one stage per tick
for every job in flight, budget released only when a job's MSMs complete,
and the latency percentiles.
"""

from __future__ import annotations

import numpy as np
import pytest

from zkgpu.prover import STAGE_COSET, STAGE_DONE, STAGE_INTT, STAGE_MSM, STAGE_QUOTIENT, vanishing_inverse
from zkgpu.curve import R
from zkgpu.serving import JobRecord, Scheduler, percentile, summarize


def test_admission_is_fifo_under_the_budget():
    s = Scheduler(hbm_budget=100)
    for k, (fp, t) in enumerate([(40, 0.0), (40, 0.0), (40, 0.1), (10, 0.1)]):
        s.submit(k, fp, t)
    assert s.admit(0.05) == [0, 1]  # job 2 has not arrived yet
    assert s.admit(0.2) == []  # job 2 does not fit; job 3 would, but waits its turn
    s.next_tick()
    for _ in range(3):
        s.next_tick()
    assert s.stage == {0: STAGE_DONE, 1: STAGE_DONE}
    s.finish(0)
    assert s.used == 40
    assert s.admit(0.2) == [2, 3]
    assert s.used == 90


def test_a_job_larger_than_the_budget_runs_alone():
    s = Scheduler(hbm_budget=10)
    s.submit(0, 50, 0.0)
    s.submit(1, 5, 0.0)
    assert s.admit(0.0) == [0]
    assert s.admit(0.0) == []
    for _ in range(4):
        s.next_tick()
    s.finish(0)
    assert s.admit(0.0) == [1]


def test_every_job_in_flight_advances_one_stage_per_tick():
    s = Scheduler(hbm_budget=1000)
    s.submit(0, 1, 0.0)
    s.submit(1, 1, 1.0)
    t = s.next_tick(s.admit(0.0))
    assert (t.admitted, t.intt) == ([0], [0])
    t = s.next_tick(s.admit(1.0))  # job 1 joins while job 0 is in flight
    assert (t.admitted, t.intt, t.coset) == ([1], [1], [0])
    t = s.next_tick()
    assert (t.coset, t.quotient) == ([1], [0])
    t = s.next_tick()
    assert (t.quotient, t.msm) == ([1], [0])
    assert s.stage == {0: STAGE_DONE, 1: STAGE_MSM}
    with pytest.raises(ValueError):
        s.finish(1)
    s.finish(0)
    t = s.next_tick()
    assert t.msm == [1] and not t.intt
    s.finish(1)
    assert s.idle() and s.finished == [0, 1]
    assert [STAGE_INTT, STAGE_COSET, STAGE_QUOTIENT, STAGE_MSM, STAGE_DONE] == list(range(5))


def test_submissions_must_be_in_arrival_order():
    s = Scheduler(hbm_budget=10)
    s.submit(0, 1, 1.0)
    with pytest.raises(ValueError):
        s.submit(1, 1, 0.5)
    with pytest.raises(ValueError):
        Scheduler(hbm_budget=0)


def test_percentiles_and_summary():
    rng = np.random.default_rng(0)
    v = list(rng.exponential(5.0, size=501))
    for q in (0, 50, 90, 99, 100):
        assert percentile(v, q) == pytest.approx(float(np.percentile(v, q)))
    recs = [JobRecord(k, 4096, 0.01 * k, finished_s=0.01 * k + 0.002 * (k % 5 + 1)) for k in range(100)]
    out = summarize(recs)
    assert out["jobs"] == 100
    assert out["p50_ms"] == pytest.approx(6.0)
    assert out["max_ms"] == pytest.approx(10.0)


def test_vanishing_inverse():
    for m in (4, 4096, 1 << 20):
        assert vanishing_inverse(m) * (pow(5, m, R) - 1) % R == 1
