"""
bench.py's host logic without a GPU: the multi-rank plumbing (barrier and the
max over ranks) as two gloo processes on the CPU, the reference arm's JSON
line on a tiny workload, and the GLV digit count behind the roofline.
"""

from __future__ import annotations

import os
import socket
import sys
from types import SimpleNamespace

import pytest
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    import torch

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist = bench.init_dist(world, "gloo")
    device = torch.device("cpu")
    bench.barrier(dist, device)
    worst = bench.max_over_ranks(10.0 * (rank + 1), dist, device)  # each rank reports its own time
    again = bench.max_over_ranks(-1.0 * rank, dist, device)
    ref = bench.run_reference(SimpleNamespace(workload="tiny", steps=1, warmup=0), rank, world)
    dist.destroy_process_group()
    out.put((rank, worst, again, ref is None))


def test_two_gloo_ranks_agree_on_the_max_and_only_rank0_runs_the_reference():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [20.0, 20.0]  # the slowest rank's time, on every rank
    assert [r[2] for r in results] == [0.0, 0.0]
    assert results[0][3] is False and results[1][3] is True  # rank 0 reports, rank 1 does no work


def test_reference_arm_line_follows_the_contract():
    line = bench.run_reference(SimpleNamespace(workload="tiny", steps=2, warmup=1), 0, 1)
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["unit"] == "ms" and line["higher_is_better"] is False and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] == os.cpu_count()
    assert line["e2e"] == {"value": line["value"], "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_nonzero_digit_count_matches_the_recoding():
    import numpy as np

    from zkgpu import workloads as wl

    k = np.array([[0, 0, 0, 0], [1, 0, 0, 0], [2**32 - 1, 0, 0, 0]], dtype=np.uint64)
    # 0 has no digits; 1 is one digit; 2^32 - 1 at w = 16 recodes to -1 + 0 * 2^16 + 1 * 2^32
    assert bench.nonzero_digits(k, 16) == 0 + 1 + 2
    u = wl.uniform_fr(3, 512)
    n = bench.nonzero_digits(u, 16)
    assert 2 * 8 * 512 * 0.99 < n <= 2 * 8 * 512  # nearly every digit of both GLV halves is nonzero


@pytest.mark.parametrize("w", [1, 5, 13, 16])
def test_glv_halves_recombine(w):
    from oracle import pyoracle as po
    from zkgpu import workloads as wl

    lam = 0xB3C4D79D41A917585BFC41088D8DAAA78B17EA66B99C90DD
    for k in wl.rows_to_ints(wl.uniform_fr(w, 64)):
        a, b = bench._glv_halves(k)
        assert a < 2**127 and b < 2**127
        c1, c2 = (k * bench._GLV_G1) >> 256, (k * bench._GLV_G2) >> 256
        k1 = k - c1 * bench._GLV_A1 - c2 * bench._GLV_A2
        k2 = c1 * bench._GLV_B1_ABS - c2 * bench._GLV_A1
        assert (k1 + k2 * lam - k) % po.R == 0


def test_ntt_product_count_follows_the_pass_plan():
    """Products per row of the NTT the roofline counts: 12 radix-4 rounds over two 12-bit passes
    (11.5 per row at 2^24) or three 8-bit passes (11.75), the default plan from 2^19 rows."""
    n = 1 << 24
    assert bench.ntt_products(n, 24, 2) == int(11.5 * n)
    assert bench.ntt_products(n, 24, 3) == int(11.75 * n)
    assert bench.ntt_products(n, 24) == bench.ntt_products(n, 24, 3)
    assert bench.ntt_products(1 << 16, 16) == bench.ntt_products(1 << 16, 16, 2) == int(7.5 * (1 << 16))
    assert bench.ntt_products(1 << 9, 9) == int(((0.25 + 3) + 0.5) * (1 << 9))  # one pass, odd radix


def test_gpus_flag_starts_one_rank_per_gpu_without_a_launcher():
    """`bench.py --gpus 2` with no torchrun environment starts two ranks itself; rank 0
    prints the line and sees both ranks (gloo here, NCCL on GPUs)."""
    import json
    import subprocess

    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_PORT")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--check-ranks"], env=env,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["gpus_requested"] == 2 and line["backend"] == "gloo"
    assert line["ranks"] == [[0, 0], [1, 1]]
    assert line["max_over_ranks"] == 2.0


def test_gpus_flag_must_match_the_launcher():
    import subprocess

    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0", CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--check-ranks"], env=env,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode != 0 and "--gpus 2" in out.stderr


def test_reference_arm_times_every_requested_step_and_hashes_its_outputs():
    from oracle import c_oracle as co
    from zkgpu import workloads as wl

    line = bench.run_reference(SimpleNamespace(workload="tiny", steps=4, warmup=1), 0, 1)
    assert line["steps"] == 4 and line["steps_timed"] == 4
    assert line["config"] == bench.workload_config(10, 10, 1)
    # the digest is that of the C port's outputs on the seeded inputs
    n = 1 << 10
    bases = co.mul_generator(wl.base_scalars(10, n), threads=2)
    ntt_h = co.to_mont(co.FR, wl.uniform_fr(13, n))
    outs, _ = bench.oracle_outputs(bases, wl.uniform_fr(11, n), wl.skewed_scalars(12, n), ntt_h, 2)
    assert line["outputs_sha256"] == bench.outputs_sha256(*outs)
