"""
Groth16-shaped prover jobs on the GPU (zkgpu.prover, zkgpu.serving): one job's
quotient and four MSMs against the C oracle (the reference's algorithms:
inverse NTT, coset NTT, pointwise, inverse coset NTT, Pippenger), and every
job served in a mix of concurrent jobs of different sizes equal to the same
job run alone.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import c_oracle as co
from zkgpu import curve_gpu
from zkgpu import workloads as wl
from zkgpu.curve import Point
from zkgpu.prover import COSET, MSM_NAMES, ProofJob, prove_plain, synthetic_request, vanishing_inverse
from zkgpu.serving import Server, summarize

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bases():
    return curve_gpu.mul_generator(wl.base_scalars(7, 1 << 15))


def _oracle_job(req, bases_host):
    """h and the four MSM points of one job by the C oracle."""
    threads = os.cpu_count() or 1
    m = req.m
    rows = [co.to_mont(co.FR, v) for v in (req.a, req.b, req.c)]
    coef = [co.ntt(r, invert=True, threads=threads) for r in rows]
    ev = [co.ntt(c, coset=COSET, threads=threads) for c in coef]
    z = co.to_mont(co.FR, np.array([[(vanishing_inverse(m) >> (64 * j)) & (2**64 - 1) for j in range(4)]] * m,
                                   dtype=np.uint64))
    q = co.field_op("mul", co.FR, co.field_op("sub", co.FR, co.field_op("mul", co.FR, ev[0], ev[1]), ev[2]), z)
    h = co.from_mont(co.FR, co.ntt(q, invert=True, coset=COSET, threads=threads))
    w = 10
    scal = {"A": req.witness, "B": req.witness, "L": req.witness[2:], "H": h[: m - 1]}
    pts = {}
    for name in MSM_NAMES:
        s = scal[name]
        out = co.msm(bases_host[: s.shape[0]], s, w, threads=threads)
        pts[name] = Point.identity() if out[8] else Point(*wl.rows_to_ints(out[:8].reshape(2, 4)))
    return h, pts


def test_one_job_matches_the_oracle(bases):
    req = synthetic_request(11, 1 << 12)
    job = ProofJob(req, bases)
    prove_plain(job)
    job.check_quotient()
    h, pts = _oracle_job(req, bases.cpu().numpy())
    assert np.array_equal(job.h_plain.cpu().numpy().view(np.uint64), h)
    assert not h[-1].any()  # degree <= m - 2: the circuit is satisfied
    assert job.msm_points() == pts


def test_served_jobs_equal_the_same_jobs_alone(bases):
    import torch

    reqs = [synthetic_request(20 + k, m) for k, m in enumerate([1 << 12, 1 << 14, 1 << 12, 1 << 13, 1 << 15, 1 << 12])]
    alone = []
    for r in reqs:
        job = ProofJob(r, bases)
        prove_plain(job)
        torch.cuda.synchronize()
        job.check_quotient()
        alone.append((job.h_plain.cpu().numpy().copy(), job.msm_points()))
    # a mix: jobs arrive 1 ms apart, so several are in flight at different stages; a small
    # budget also makes some wait for others to finish
    server = Server(bases, hbm_budget=200 << 20)
    keep = {}
    orig_collect = server._collect

    def collect(block):  # keep each job's outputs before the server drops it
        for job_id, job in list(server.jobs.items()):
            keep[job_id] = job
        orig_collect(block)

    server._collect = collect
    recs = server.run(reqs + reqs[:2], [0.001 * k for k in range(len(reqs) + 2)])
    assert len(recs) == len(reqs) + 2 and all(r.finished_s >= r.arrival_s for r in recs)
    for job_id, job in keep.items():
        want_h, want_pts = alone[job_id % len(reqs)]
        assert np.array_equal(job.h_plain.cpu().numpy(), want_h), job_id
        assert job.msm_points() == want_pts, job_id
    assert len(keep) == len(reqs) + 2
    s = summarize(recs)
    assert s["p99_ms"] >= s["p50_ms"] > 0
    assert server.ticks >= 4 and server.launches > 0


def test_many_jobs_admitted_at_once_upload_in_groups(bases):
    """30 jobs queued at once: one tick admits them all, so their rows go up in two copy groups
    (21 + 9 jobs, each group's work waiting only for its own copies); a second server on the same
    streams then reuses the memory the first one freed. Every job equals the same job alone."""
    import torch

    pool = [synthetic_request(60 + k, m) for k, m in enumerate([1 << 12, 1 << 13, 1 << 12, 1 << 14])]
    alone = []
    for r in pool:
        job = ProofJob(r, bases)
        prove_plain(job)
        torch.cuda.synchronize()
        alone.append((job.h_plain.cpu().numpy().copy(), job.msm_points()))
    reqs = [pool[k % len(pool)] for k in range(30)]
    for _ in range(2):
        server = Server(bases, hbm_budget=60 << 30)
        keep = {}
        orig_collect = server._collect

        def collect(block, server=server, keep=keep, orig=orig_collect):
            for job_id, job in list(server.jobs.items()):
                keep[job_id] = job
            orig(block)

        server._collect = collect
        recs = server.run(reqs, [0.0] * len(reqs))
        assert len(recs) == len(reqs) and len(keep) == len(reqs)
        for job_id, job in keep.items():
            want_h, want_pts = alone[job_id % len(pool)]
            assert np.array_equal(job.h_plain.cpu().numpy(), want_h), job_id
            assert job.msm_points() == want_pts, job_id
