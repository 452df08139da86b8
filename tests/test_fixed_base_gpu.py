"""
MSMs over fixed-base tables (zkgpu.msm_gpu.FixedBaseTable, zkb_msm_table_build,
zkb_msm_fixed_batch): the per-window multiples of a resident base set. The
reference has no such path; its MSM takes the points with every call. So every
case here is checked against the reference's own answers (the golden seeded
MSMs) or against the regular MSM over the same points, at table windows 8 to
24, over prefixes of the table, in batches, and inside the prover and server.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, hs
from oracle import pyoracle as po
from zkgpu import batch, curve_gpu, msm_gpu
from zkgpu import workloads as wl
from zkgpu.curve import Point
from zkgpu.msm_gpu import FixedBaseTable

pytestmark = pytest.mark.gpu


def expected_point(case) -> Point:
    return Point.identity() if case["expected"] is None else Point(*hs(case["expected"]))


def _bases(n: int, seed: int):
    return curve_gpu.mul_generator(wl.base_scalars(seed, n))


@pytest.mark.parametrize("w", [8, 13, 16, 20, 24])
def test_table_msm_gives_the_references_points(w):
    for case in golden("msm.json")["seeded"][:2]:
        n = case["n"]
        bases = _bases(n, case["base_seed"])
        gen = wl.uniform_fr if case["kind"] == "uniform" else wl.skewed_scalars
        sc = gen(case["scalar_seed"], n)
        assert FixedBaseTable(bases, w).msm(sc) == expected_point(case), (case["kind"], w)


def test_a_table_serves_every_prefix_and_batches():
    import torch

    bases = _bases(1 << 14, 5)
    table = FixedBaseTable(bases, 16)
    sizes = [0, 1, 2, 100, 4096, 1 << 14, 777]
    scs = [torch.from_numpy(wl.skewed_scalars(40 + k, n)).cuda() for k, n in enumerate(sizes)]
    want = batch.msm_batch([bases[:n] for n in sizes], scs)
    assert batch.msm_fixed_batch(table, scs) == want
    assert [table.msm(s) for s in scs] == want


def test_edge_scalars_over_a_table():
    import torch

    pts = [po.scalar_mul(po.G, k) for k in range(1, 301)]
    rows = curve_gpu.mul_generator(np.array([[k, 0, 0, 0] for k in range(1, 301)], dtype=np.uint64))
    table = FixedBaseTable(rows, 12)
    r = 21888242871839275222246405745257275088548364400416034343698204186575808495617
    cases = {
        "heavy bucket": [2**200 + 12345] * 300,
        "booleans": [int(k % 3 != 0) for k in range(300)],
        "zeros": [0] * 300,
        "r and beyond": [r, r + 5, 2**256 - 1] + [7] * 297,
        "negatives mod r": [r - k for k in range(1, 301)],
    }
    for name, scalars in cases.items():
        limbs = np.array([[(s >> (64 * j)) & (2**64 - 1) for j in range(4)] for s in scalars], dtype=np.uint64)
        got = table.msm(torch.from_numpy(limbs).cuda())
        want = po.msm_double_and_add(pts, [s % r for s in scalars])
        assert got == (Point.identity() if want is None else Point(*want)), name


def test_invalid_tables_and_jobs_are_refused():
    import torch

    bases = _bases(64, 3)
    with pytest.raises(ValueError, match="window_size"):
        FixedBaseTable(bases, 7)
    with pytest.raises(ValueError, match="window_size"):
        FixedBaseTable(bases, 25)
    table = FixedBaseTable(bases, 16)
    too_many = torch.from_numpy(wl.uniform_fr(1, 65)).cuda()
    with pytest.raises(ValueError, match="table of 64"):
        table.msm(too_many)


def test_served_jobs_over_a_table_equal_the_jobs_alone():
    import torch

    from zkgpu.prover import ProofJob, prove_plain, synthetic_request
    from zkgpu.serving import Server

    bases = _bases(1 << 15, 7)
    table = FixedBaseTable(bases, 16)
    reqs = [synthetic_request(60 + k, m) for k, m in enumerate([1 << 12, 1 << 15, 1 << 13, 1 << 12])]
    alone = []
    for r in reqs:
        job = ProofJob(r, bases)
        prove_plain(job)
        torch.cuda.synchronize()
        alone.append(job.msm_points())
        job_t = ProofJob(r, bases)
        prove_plain(job_t, table=table)
        torch.cuda.synchronize()
        assert job_t.msm_points() == alone[-1]
    server = Server(bases, hbm_budget=400 << 20, table=table)
    keep = {}
    orig_collect = server._collect

    def collect(block):
        for job_id, job in list(server.jobs.items()):
            keep[job_id] = job
        orig_collect(block)

    server._collect = collect
    recs = server.run(reqs, [0.001 * k for k in range(len(reqs))])
    assert len(recs) == len(reqs)
    for job_id, job in keep.items():
        assert job.msm_points() == alone[job_id], job_id


def test_full_batches_of_64_jobs():
    """The largest batch (64 jobs) through the counting-sort pipeline and over a table: sizes
    from 0 to 2^11, uniform and skewed scalars, against one MSM per job."""
    import torch

    bases = _bases(1 << 11, 9)
    table = FixedBaseTable(bases, 10)
    rng = np.random.default_rng(3)
    sizes = [0, 1] + [int(v) for v in rng.integers(2, 1 << 11, size=62)]
    scs = []
    for k, n in enumerate(sizes):
        gen = wl.uniform_fr if k % 2 else wl.skewed_scalars
        scs.append(torch.from_numpy(gen(500 + k, n) if n else np.zeros((0, 4), dtype=np.uint64)).cuda())
    one_by_one = [msm_gpu.msm_pippenger_rows(bases[:n], s, check_points=False) if n else Point.identity()
                  for n, s in zip(sizes, scs, strict=True)]
    assert batch.msm_batch([bases[:n] for n in sizes], scs) == one_by_one
    assert batch.msm_fixed_batch(table, scs) == one_by_one
