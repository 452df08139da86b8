"""
Full-size parity of exactly what bench.py times: the large workload's step
(MSM over 2^22 points with uniform and with skewed scalars, an Fr NTT of 2^24
rows and its coset form), built and run as the bench runs it (bench.Step: one
MSM batch on a high-priority stream, both transforms beside it on a
low-priority stream), on the bench's seeds, compared bit for bit with the C
port of the reference's CPU algorithms (oracle/zk_oracle.c) on all host
threads. The one-call forms (zkb_msm, zkb_ntt) are compared too, and the
step's SHA-256 equals the oracle's, as the two arms of the bench print them.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from conftest import ROOT
from oracle import c_oracle as co
from zkgpu import workloads as wl

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402

pytestmark = pytest.mark.gpu


def test_bench_step_matches_the_oracle_at_full_size():
    import torch

    step = bench.Step(22, 24, seed=10)
    # the bases the GPU made for the bench (k_i G) against the oracle on a seeded subset
    sub = np.ascontiguousarray(step.k_host[: 1 << 12])
    assert np.array_equal(step.bases[: 1 << 12].cpu().numpy(), co.mul_generator(sub, threads=os.cpu_count() or 1))
    step.plan.run()
    for _, fn in step.parts():
        fn()
    torch.cuda.synchronize()
    plan_outs = [step.plan.msm_results[0, :9].cpu().numpy().view(np.uint64),
                 step.plan.msm_results[1, :9].cpu().numpy().view(np.uint64),
                 step.plan.ntt_outputs[0].cpu().numpy(), step.plan.ntt_outputs[1].cpu().numpy()]
    outs, _ = bench.oracle_outputs(step.bases.cpu().numpy(), step.sc_uniform_host, step.sc_skewed_host,
                                   step.ntt_in.cpu().numpy(), os.cpu_count() or 1)
    names = ("msm uniform", "msm skewed", "ntt", "coset ntt")
    for name, a, b in zip(names[:2], outs[:2], plan_outs[:2]):
        assert np.array_equal(np.asarray(a, dtype=np.uint64)[:9], b), name
    for name, a, b in zip(names[2:], outs[2:], plan_outs[2:]):
        assert np.array_equal(np.asarray(a).view(np.uint64), b.view(np.uint64)), name
    assert bench.outputs_sha256(*plan_outs) == bench.outputs_sha256(*outs)
    # the one-call forms: zkb_msm into step.result, and the skewed MSM / NTTs again
    assert np.array_equal(step.result[0, :9].cpu().numpy().view(np.uint64), plan_outs[0])
    assert np.array_equal(step.result[1, :9].cpu().numpy().view(np.uint64), plan_outs[1])
    assert step.same_results()
    # the inputs are the bench's seeds (10 bases, 11 uniform, 12 skewed, 13 NTT)
    assert np.array_equal(step.sc_uniform_host, wl.uniform_fr(11, 1 << 22))
    assert np.array_equal(step.sc_skewed_host, wl.skewed_scalars(12, 1 << 22))
