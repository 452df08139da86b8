"""
bench.py — the BN254 prover hot path on B200: large plain instances.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload large|small]

Workload "large" (default; the headline metric is quoted on it): one step =
  MSM over 2^22 BN254 G1 points with uniform scalars
  + the same MSM with skewed witness-like scalars (60% in {0,1}, 20% < 2^32)
  + a forward Fr NTT of 2^24 elements
  + a forward coset NTT (g = 5) of 2^24 elements.
Inputs are seeded synthetic data with the configs' shapes (bases k_i G, k_i
uniform in [1, r)); every input is larger than the 126 MB L2.

Prints ONE JSON line (rank 0). `value` is device time per step with inputs
resident in HBM (CUDA events, max over ranks); `e2e` is the same step through
the public Python API from pinned host buffers, copies included; `roofline`
covers the dominant kernel (the MSM bucket accumulation, integer-multiply
bound) timed live with CUDA events recorded by the library on its stream;
`cpu_baseline` is the oracle (a C port of the reference's CPU algorithms)
timed on a bounded sample on one host core.

Two more objects on the line cover the rest of the metric ("batched jobs/s
vs plain launches; p99 latency"), on the large workload only:
`batched` — 64 NTTs + 32 MSMs of uneven sizes as one batch (one persistent
NTT launch, one MSM batch, and its CUDA-graph replay) against one call per
job; `served` — a Poisson stream of 2,000 Groth16-shaped prover jobs through
the continuous-batching server, with p50/p99 latency, against the same jobs
one at a time. `int64` — the int64-field path (moduli below 2^63): a 2^25-word
NTT and a 2^26-word element-wise product, with their HBM rooflines.

--impl reference runs the reference's CPU algorithms (the same C port, all
host threads) on the same workload and prints the same line with
"impl": "reference". Both arms print `outputs_sha256`, a digest of the step's
four results, and our arm checks the timed results bit for bit against the
C port at full size (`parity_full`).

N > 1: under torchrun, or started here when --gpus N > 1 and no launcher set
WORLD_SIZE (one process per GPU, rendezvous on 127.0.0.1). Every rank runs
its own instance of the step (weak scaling, no collective on the data path);
the time is the max over ranks. Beside it, `sharded` times one MSM and one
NTT split over the ranks (strong scaling, NCCL exchanges). --check-ranks runs
only the multi-rank plumbing (gloo on a machine without GPUs).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "zk-gpu-accelerator_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "MSM 2^22 / NTT 2^24 ms on 1 B200; batched jobs/s vs plain launches; p99 latency"
UNIT = "ms"
SCALAR_BITS = 254
COSET = 5

WORKLOADS = {
    # name: (log2 MSM points, log2 NTT size)
    "large": (22, 24),
    "small": (20, 22),  # for profiler captures: inputs above the L2 size, ~2 GB on the device
    "medium": (21, 23),  # for profiler captures whose point set (bases + phi images, 256 MB) exceeds L2
    "tiny": (10, 10),   # for the CPU tests of the reference arm
}


def workload_config(log_msm: int, log_ntt: int, world: int) -> dict:
    """The `config` object of both arms' lines: what the step computes, on which inputs
    (implementation choices such as the window go under `impl_config`)."""
    return {"workload": f"msm-2^{log_msm}-uniform+skewed, ntt-2^{log_ntt}+coset",
            "msm_points": 1 << log_msm, "ntt_size": 1 << log_ntt, "coset": COSET,
            "scalars": ["uniform [0,r)", "skewed 60% {0,1} / 20% < 2^32 / 20% uniform"],
            "seeds": {"bases": 10, "uniform": 11, "skewed": 12, "ntt": 13, "per_rank_offset": 100},
            "l2": "every input larger than the 126 MB L2 (bases 256 MiB, NTT 512 MiB)"
                  if log_msm >= 22 else "small inputs",
            "parallelism": f"replicas x{world}"}


def outputs_sha256(msm_uniform, msm_skewed, ntt_plain, ntt_coset) -> str:
    """SHA-256 over one step's results: the two MSM results as 9 little-endian uint64 each
    (plain affine x, y, then the infinity flag) and the two transforms' Montgomery rows.
    Both arms hash the same bytes, so equal digests mean identical outputs."""
    import hashlib

    import numpy as np

    h = hashlib.sha256()
    for a in (msm_uniform, msm_skewed):
        h.update(np.ascontiguousarray(np.asarray(a, dtype=np.uint64).reshape(-1)[:9]).tobytes())
    for a in (ntt_plain, ntt_coset):
        h.update(np.ascontiguousarray(np.asarray(a).view(np.uint64)).tobytes())
    return h.hexdigest()


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            pass
    return {}


# ------------------------------------------------------------------
# Work accounting
# ------------------------------------------------------------------

IMAD_PER_MULMOD = 264  # 2 x 64 32-bit multiply-adds (lo and hi) for a*b and m*p, plus 8 for the m's
IMAD_PER_SQR = 208     # 2 x (36 + 64) for a*a (each cross product once) and m*p, plus 8 for the m's
# XYZZ mixed addition: 8 multiplications + 2 squarings
IMAD_PER_MADD = 8 * IMAD_PER_MULMOD + 2 * IMAD_PER_SQR
PRODUCTS_PER_MADD = 10


# GLV split constants (csrc/msm.cu): k = k1 + k2 lambda, c1 = floor(k g1 / 2^256), ...
_R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
_GLV_A1 = 9931322734385697763
_GLV_B1_ABS = 147946756881789319000765030803803410728
_GLV_A2 = 147946756881789319010696353538189108491
_GLV_G1 = 0x2D91D232EC7E0B3D7
_GLV_G2 = 0x24CCEF014A773D2CF7A7BD9D4391EB18E


def ntt_products(n: int, log_n: int, passes: int | None = None) -> int:
    """Montgomery products of one forward NTT of n = 2^log_n rows as csrc/ntt.cu runs it: log_n
    split evenly into P passes (`passes`, else the library's default plan: three from 2^19, else
    at most 12 bits each and two from 2^10); a pass of 2^lr rows does lr / 2 radix-4 rounds, the
    first with only the w_4 product (1 per 4 rows), the others 4 per 4 rows, plus a radix-2 stage
    (1 per 2 rows) for odd lr; each pass boundary 1 product per row (the twiddle read from the
    expanded table)."""
    P = passes or (3 if log_n >= 19 else max(-(-log_n // 12), 2 if log_n >= 10 else 1))
    radices = [log_n // P + (1 if q < log_n % P else 0) for q in range(P)]
    per_row = 0.0
    for lr in radices:
        rounds = lr // 2
        per_row += (0.25 + (rounds - 1) if rounds else 0.0) + (0.5 if lr % 2 and lr > 1 else 0.0)
    per_row += P - 1
    return int(per_row * n)


def _glv_halves(k: int) -> tuple[int, int]:
    c1, c2 = (k * _GLV_G1) >> 256, (k * _GLV_G2) >> 256
    return abs(k - c1 * _GLV_A1 - c2 * _GLV_A2), abs(c1 * _GLV_B1_ABS - c2 * _GLV_A1)


def nonzero_digits(scalars, w: int, sample: int = 1 << 16) -> int:
    """Mixed additions the bucket kernel performs: nonzero signed w-bit digits of
    both GLV halves (csrc/msm.cu's recoding: ceil(128 / w) windows, a digit above
    2^(w-1) borrows). Counted exactly on the first `sample` scalars, scaled to n."""
    import numpy as np

    from zkgpu import workloads as wl

    n = scalars.shape[0]
    m = min(n, sample)
    W = -(-128 // w)
    half = 1 << (w - 1)
    mask = (1 << w) - 1
    count = 0
    for k in wl.rows_to_ints(np.ascontiguousarray(scalars[:m])):
        for v in _glv_halves(k % _R):
            carry = 0
            for win in range(W):
                raw = ((v >> (win * w)) & mask) + carry
                if win + 1 < W and raw > half:
                    mag, carry = (1 << w) - raw, 1
                else:
                    mag, carry = raw, 0
                count += mag != 0
    return round(count * n / m)


# ------------------------------------------------------------------
# Clocks (nvidia-smi sampled during the timed region)
# ------------------------------------------------------------------

CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    def __init__(self, gpu_index: int) -> None:
        self.gpu = gpu_index
        self.proc: subprocess.Popen | None = None
        self.lines: list[str] = []
        self._t: threading.Thread | None = None

    def __enter__(self) -> ClockSampler:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={CLOCK_QUERY}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self) -> None:
        assert self.proc and self.proc.stdout
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc) -> None:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self._t:
            self._t.join(timeout=2)

    def summary(self) -> dict:
        rows = []
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append({"sm": float(parts[1]), "max": float(parts[2]), "power": float(parts[3]),
                             "hw": parts[5], "hw_thermal": parts[6], "sw_thermal": parts[7], "sw_power": parts[8]})
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        loaded = [r for r in rows if r["power"] > 0.5 * max(r["power"] for r in rows)] or rows
        reasons = []
        for key, name in (("hw", "hw_slowdown"), ("hw_thermal", "hw_thermal_slowdown"),
                          ("sw_thermal", "sw_thermal_slowdown"), ("sw_power", "sw_power_cap")):
            if any(r[key].lower() == "active" for r in rows):
                reasons.append(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in loaded), "sm_max_mhz": max(r["max"] for r in rows),
                "reasons": reasons, "samples": len(rows), "power_w_max": max(r["power"] for r in rows)}


# ------------------------------------------------------------------
# Distributed plumbing
# ------------------------------------------------------------------


def dist_env() -> tuple[int, int, int]:
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def _free_port() -> int:
    import socket

    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def spawn_ranks(n: int, argv: list[str], timeout_s: float | None = None) -> int:
    """`python bench.py --gpus N` without a launcher: start N copies of this script as
    ranks 0..N-1 (one per GPU, LOCAL_RANK = RANK) with the torch.distributed rendezvous
    on 127.0.0.1, pass rank 0's output through, and return the worst exit code. If a rank
    fails, the others are stopped (by their own process handles) instead of waiting on a
    collective that will not complete."""
    port = _free_port()
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(Path(__file__).resolve()), *argv], env=env,
                                      stdout=None if r == 0 else subprocess.DEVNULL))
    deadline = None if timeout_s is None else time.monotonic() + timeout_s
    codes: dict[int, int] = {}
    while len(codes) < n:
        for r, p in enumerate(procs):
            if r not in codes and p.poll() is not None:
                codes[r] = p.returncode
        if any(c != 0 for c in codes.values()) or (deadline is not None and time.monotonic() > deadline):
            for r, p in enumerate(procs):
                if r not in codes:
                    p.kill()
                    codes[r] = p.wait() or 1
            break
        time.sleep(0.05)
    return max(abs(c) for c in codes.values())


def check_ranks(args, rank: int, world: int, local_rank: int) -> dict | None:
    """The multi-rank plumbing alone (process group, barrier, max over ranks, a gather
    of every rank's identity), on the GPUs with NCCL or on the CPU with gloo."""
    import torch

    cuda = torch.cuda.is_available()
    if cuda:
        torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank) if cuda else torch.device("cpu")
    dist = init_dist(world, "nccl" if cuda else "gloo")
    barrier(dist, device)
    worst = max_over_ranks(float(rank + 1), dist, device)
    ident = torch.tensor([rank, local_rank, os.getpid()], dtype=torch.int64, device=device)
    if dist is not None:
        everyone = [torch.zeros_like(ident) for _ in range(world)]
        dist.all_gather(everyone, ident)
        dist.destroy_process_group()
    else:
        everyone = [ident]
    if rank != 0:
        return None
    return {"check": "ranks", "n_gpus": world, "gpus_requested": args.gpus, "backend": "nccl" if cuda else "gloo",
            "ranks": [[int(v) for v in t.tolist()[:2]] for t in everyone], "max_over_ranks": worst}


def init_dist(world: int, backend: str):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=180))
    return dist


def max_over_ranks(value: float, dist, device) -> float:
    """The largest value any rank reports (all ranks call this in the same order)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device) -> None:
    if dist is not None:
        import torch

        dist.barrier(device_ids=[device.index] if device is not None and device.type == "cuda" else None)


# ------------------------------------------------------------------
# Our implementation
# ------------------------------------------------------------------


class Step:
    """One step's device buffers and launches through the C ABI (inputs resident in HBM)."""

    def __init__(self, log_msm: int, log_ntt: int, seed: int) -> None:
        import numpy as np
        import torch

        from zkgpu import _native, curve_gpu, workloads as wl
        from zkgpu.field256_gpu import BN254_FR

        self.torch, self.np, self.native, self.wl = torch, np, _native, wl
        self.lib = _native.lib()
        self.n, self.m = 1 << log_msm, 1 << log_ntt
        n, m = self.n, self.m
        self.k_host = wl.base_scalars(seed, n)
        self.bases = curve_gpu.mul_generator(self.k_host)  # (n, 2, 4) Montgomery, resident
        self.sc_uniform_host = wl.uniform_fr(seed + 1, n)
        self.sc_skewed_host = wl.skewed_scalars(seed + 2, n)
        self.sc_uniform = torch.from_numpy(self.sc_uniform_host).cuda()
        self.sc_skewed = torch.from_numpy(self.sc_skewed_host).cuda()
        self.ntt_plain_host = wl.uniform_fr(seed + 3, m)
        self.ntt_in = BN254_FR.to_montgomery(self.ntt_plain_host)
        self.ntt_out = torch.empty_like(self.ntt_in)
        self.field = BN254_FR._field()
        self.w = int(self.lib.zkb_msm_default_window(n))
        self.msm_ws_bytes = int(self.lib.zkb_msm_workspace_bytes(n, self.w))
        self.msm_ws = torch.empty(self.msm_ws_bytes, dtype=torch.uint8, device="cuda")
        self.ntt_ws_bytes = int(self.lib.zkb_ntt_workspace_bytes(m))
        self.ntt_ws = torch.empty(max(self.ntt_ws_bytes, 1), dtype=torch.uint8, device="cuda")
        self.result = torch.empty((2, 16), dtype=torch.int64, device="cuda")  # 128-byte rows
        self.coset = _native.u64_array(_native.limbs(COSET))
        # the step as one job: both MSMs in one MSM batch, both NTTs in one persistent
        # NTT launch on a side stream beside it
        from zkgpu.batch import BatchPlan

        self.plan = BatchPlan(ntt_jobs=[(self.ntt_in, False, None), (self.ntt_in, False, COSET)],
                              msm_jobs=[(self.bases, self.sc_uniform, self.w), (self.bases, self.sc_skewed, self.w)],
                              concurrent=True)
        torch.cuda.synchronize()

    def same_results(self) -> bool:
        """The batched step's results equal the one-call results (run both first)."""
        from zkgpu.field256_gpu import BN254_FR

        t = self.torch
        msm_same = bool((self.plan.msm_results[:2, :9] == self.result[:, :9]).all())
        fwd = BN254_FR.ntt(self.ntt_in)
        cos = BN254_FR.ntt(self.ntt_in, coset=COSET)
        t.cuda.synchronize()
        return msm_same and bool((self.plan.ntt_outputs[0] == fwd).all()) and \
            bool((self.plan.ntt_outputs[1] == cos).all())

    def msm(self, scalars, out_row: int) -> None:
        s = self.native.stream_ptr()
        self.native.check(self.lib.zkb_msm(
            self.bases.data_ptr(), scalars.data_ptr(), self.n, self.w, self.result[out_row].data_ptr(),
            self.msm_ws.data_ptr(), self.msm_ws_bytes, s))

    def ntt(self, coset: bool) -> None:
        s = self.native.stream_ptr()
        self.native.check(self.lib.zkb_ntt(
            self.field, self.ntt_in.data_ptr(), self.ntt_out.data_ptr(), self.m, 0, None,
            self.coset if coset else None, self.ntt_ws.data_ptr(), self.ntt_ws_bytes, s))

    def parts(self):
        return (("msm_uniform", lambda: self.msm(self.sc_uniform, 0)),
                ("msm_skewed", lambda: self.msm(self.sc_skewed, 1)),
                ("ntt", lambda: self.ntt(False)),
                ("coset_ntt", lambda: self.ntt(True)))


def run_ours(args, rank: int, world: int, local_rank: int) -> dict | None:
    import numpy as np
    import torch

    from zkgpu import _native, msm_gpu
    from zkgpu.field256_gpu import BN254_FR

    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    dist = init_dist(world, "nccl")
    log_msm, log_ntt = WORKLOADS[args.workload]
    for kv in args.knob:  # library tuning knobs, before anything plans its work
        key, _, value = kv.partition("=")
        _native.tune_set(key.strip(), int(value))
    tuned = None
    if args.tune:
        from zkgpu import autotune

        t0 = time.perf_counter()
        table = autotune.autotune(range(10, log_msm + 1), range(10, log_ntt + 1))
        tuned = {"seconds": round(time.perf_counter() - t0, 1), "device": table["device"],
                 "msm_window": {int(k): v["window"] for k, v in table["msm"].items()},
                 "ntt_radix_tile_threads": {int(k): [v["max_log_radix"], v["cta_log_elems"], v["threads"]]
                                            for k, v in table["ntt"].items()}}
    step = Step(log_msm, log_ntt, seed=10 + 100 * rank)

    for _ in range(args.warmup):
        step.plan.run()
    for _, fn in step.parts():  # builds the one-call path's tables too
        fn()
    torch.cuda.synchronize()

    # ---- timed region: device time per step, inputs resident in HBM
    launches0 = int(_native.lib().zkb_launch_count())
    barrier(dist, device)
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record()
        # the library records a CUDA event pair around each stage on the stage's own stream
        # (about twenty records per step): the live timing of the dominant kernel
        _native.profile_enable(True)
        for _ in range(args.steps):
            step.plan.run()
        stop.record()
        torch.cuda.synchronize()
    prof_live = _native.profile_report()
    _native.profile_enable(False)
    barrier(dist, device)
    launches = int(_native.lib().zkb_launch_count()) - launches0
    elapsed = start.elapsed_time(stop)
    ms_step = max_over_ranks(elapsed / args.steps, dist, device)

    # ---- the same four parts one call after another, each timed (diagnostics)
    parts = step.parts()
    reps = max(2, min(args.steps, 5))
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(parts) + 1)] for _ in range(reps)]
    for k in range(reps):
        ev[k][0].record()
        for j, (_, fn) in enumerate(parts):
            fn()
            ev[k][j + 1].record()
    torch.cuda.synchronize()
    part_ms = {name: sum(ev[k][j].elapsed_time(ev[k][j + 1]) for k in range(reps)) / reps
               for j, (name, _) in enumerate(parts)}
    same = step.same_results()
    # the timed step's own outputs (the batched step's results), hashed as the reference arm hashes its own
    plan_outs = [step.plan.msm_results[0, :9].cpu().numpy().view(np.uint64),
                 step.plan.msm_results[1, :9].cpu().numpy().view(np.uint64),
                 step.plan.ntt_outputs[0].cpu().numpy(), step.plan.ntt_outputs[1].cpu().numpy()]
    digest = outputs_sha256(*plan_outs)

    # ---- stage profile (library-recorded CUDA events on the launch stream), separate steps
    _native.profile_enable(True)
    for _ in range(max(2, min(args.steps, 5))):
        step.msm(step.sc_uniform, 0)
    prof_msm = _native.profile_report()
    _native.profile_enable(False)
    _native.profile_enable(True)
    for _ in range(max(2, min(args.steps, 5))):
        step.ntt(False)
    prof_ntt = _native.profile_report()
    _native.profile_enable(False)
    torch.cuda.synchronize()

    # ---- roofline of the dominant kernel: MSM bucket accumulation (integer-multiply bound)
    clk = clocks.summary()
    peaks = _peaks()
    sm_count = torch.cuda.get_device_properties(device).multi_processor_count
    # the clock sampled during the timed region; a region too short for a sample
    # takes the maximum SM clock (never a lower clock, which would inflate frac)
    mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz") or 1965.0
    imad_peak_t = sm_count * 64 * mhz * 1e6 / 1e12  # T IMAD/s at the sampled clock
    hbm_peak = peaks.get("hbm_gbs")
    madds_u = nonzero_digits(step.sc_uniform_host, step.w)
    madds_s = nonzero_digits(step.sc_skewed_host, step.w)

    def acc_roof(madds: int, prof: dict, kernel: str, traffic) -> dict:
        count, total = prof.get("msm_acc_points", (1, float("nan")))
        ms = total / max(count, 1)
        imad = madds * IMAD_PER_MADD
        achieved = imad / (ms * 1e-3) / 1e12
        acc_bytes = madds * (64 + 8) + 2 * (-(-madds // 64)) * 132  # point gathers + sorted pairs + slots
        products = madds * PRODUCTS_PER_MADD
        return {
            "kernel": kernel, "bound": "imad", "achieved": round(achieved, 3), "peak": round(imad_peak_t, 3),
            "unit": "TIMAD/s", "frac": round(achieved / imad_peak_t, 4), "traffic": traffic,
            "peak_measured": peak_measured, "frac_of_measured": round(achieved / imad_meas_t, 4),
            "products_per_s": round(products / (ms * 1e-3) / 1e9, 3),
            "products_frac_of_measured": round(products / (ms * 1e-3) / prod_meas, 4),
            "peak_source": f"nominal issue rate: {sm_count} SMs x 64 IMAD/clk x {mhz:.0f} MHz (median SM clock "
                           "sampled in the timed region)",
            "work_per_launch": f"{madds} mixed additions x (8 x {IMAD_PER_MULMOD} + 2 x {IMAD_PER_SQR}) IMAD",
            "launch_ms": round(ms, 4), "launches": count,
            "hbm": {"achieved": round(acc_bytes / (ms * 1e-3) / 1e9, 1), "peak": hbm_peak, "unit": "GB/s",
                    "frac": round(acc_bytes / (ms * 1e-3) / 1e9 / hbm_peak, 4) if hbm_peak else None,
                    "source": "measured (MEASURED_PEAKS.json)" if hbm_peak else None},
        }

    measured = _native.measure_int_peaks()
    imad_meas_t = measured["madlo_per_clk_sm"] * sm_count * mhz * 1e6 / 1e12
    prod_meas = measured["montmul_per_clk_sm"] * sm_count * mhz * 1e6  # Montgomery products / s
    peak_measured = {
        "imad_t_per_s": round(imad_meas_t, 3), "montmul_per_s": round(prod_meas / 1e9, 3),
        "unit": "T IMAD/s; G products/s", "at_mhz": mhz,
        "per_clk_sm": {k: round(measured[f"{k}_per_clk_sm"], 3) for k in ("madlo", "madwide", "montmul")},
        "probe_mhz": {k: round(measured[f"{k}_mhz"], 1) for k in ("madlo", "madwide", "montmul")},
        "source": "zkb_measure_int_peaks (csrc/peak.cu): one-wave loops of independent mad.lo.u32, "
                  "mad.wide.u32 and 256-bit Montgomery products, SM cycle counters; scaled to the clock "
                  "sampled in the timed region"}

    traffic_u = _profile_traffic("k_msm_acc_points", step.n)
    traffic_s = _profile_traffic("k_msm_acc_points_skewed", step.n)
    # the step's own launch (both MSMs' pairs, k_msm_acc_points_batch), timed live in the
    # timed region while the transforms run beside it on the low-priority stream
    roofline = acc_roof(madds_u + madds_s, prof_live,
                        "k_msm_acc_points_batch (bucket accumulation of both MSMs of the step, live)",
                        traffic_u + traffic_s if traffic_u and traffic_s else None)
    # the uniform MSM's launch alone (one call, nothing beside it)
    roofline_alone = acc_roof(madds_u, prof_msm, "k_msm_acc_points (uniform scalars, one call alone)", traffic_u)
    # NTT passes: bytes moved (read + write of 32-byte rows per pass) against HBM
    ntt_pass_ms = sum(v[1] for k, v in prof_ntt.items() if k.startswith("ntt_")) / max(2, min(args.steps, 5))
    n_passes = sum(v[0] for k, v in prof_ntt.items() if k.startswith("ntt_")) / max(2, min(args.steps, 5))
    ntt_bytes = 64 * step.m * n_passes
    ntt_gbs = ntt_bytes / (ntt_pass_ms * 1e-3) / 1e9
    ntt_mulmods = ntt_products(step.m, log_ntt, round(n_passes) or None)
    ntt_roof = {"bytes_per_launch": int(ntt_bytes), "ms": round(ntt_pass_ms, 4), "achieved_gbs": round(ntt_gbs, 1),
                "hbm_frac": round(ntt_gbs / hbm_peak, 4) if hbm_peak else None,
                "imad_frac": round(ntt_mulmods * IMAD_PER_MULMOD / (ntt_pass_ms * 1e-3) / 1e12 / imad_peak_t, 4),
                "products": ntt_mulmods, "passes": n_passes}

    # ---- end to end through the public API, pinned host buffers, copies inside the timed region
    e2e = None
    if not args.skip_e2e:
        e2e = _run_e2e(args, step, dist, device, log_msm, log_ntt)

    # Each leg below starts from an allocator holding no cached blocks of the legs before it:
    # torch keeps freed blocks per stream, and a leg that allocates on its own streams cannot
    # reuse them, so the cache of earlier legs would only push it into failed allocations and
    # the full synchronisations that release the cache (outside every timed region).
    # The batched, served and int64 forms are one-GPU forms: measured at N = 1 only, so a
    # multi-GPU run holds its GPUs for the step, the end-to-end form and the split legs.
    single = world == 1
    batched = served = None
    if single and args.workload == "large" and not args.skip_batched:
        release_cached_memory()
        batched = run_batched()
    if single and args.workload == "large" and not args.skip_served:
        release_cached_memory()
        served = run_served()
    int64 = None
    if single and args.workload == "large" and not args.skip_int64:
        release_cached_memory()
        int64 = run_int64(cpu=rank == 0 and not args.skip_cpu_baseline)

    sharded = None
    if world > 1:
        sharded = run_sharded(args, step, dist, device, rank, world, log_msm, log_ntt)

    # the CPU baseline and the full-size parity check: rank 0 at N = 1 (every rank computes the
    # same step, and its SHA-256 is on the line at every N)
    cpu = None
    if single and rank == 0 and not args.skip_cpu_baseline:
        cpu = cpu_baseline_sample(step, threads=1)
    parity = None
    if single and rank == 0 and not args.skip_parity:
        parity = full_size_parity(step, plan_outs, digest)

    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": round(ms_step, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (8x32-bit limb Montgomery, exact)", "data": "synthetic (seeded)",
        "config": workload_config(log_msm, log_ntt, world),
        "impl_config": {"msm_window": step.w,
                        "schedule": "one MSM batch (both MSMs, one pipeline) on a high-priority stream; both "
                                    "transforms as pass launches (zkb_ntt each) on a low-priority stream "
                                    "beside it",
                        **({"knobs": dict(kv.split("=", 1) for kv in args.knob)} if args.knob else {})},
        "outputs_sha256": digest,
        "parity_full": parity,
        "sharded": sharded,
        "parts_ms": {k: round(v, 3) for k, v in part_ms.items()},
        "msm_points_per_s": {k: round(step.n / (v * 1e-3)) for k, v in part_ms.items() if k.startswith("msm")},
        "sequential_ms": round(sum(part_ms.values()), 3),
        "same_as_one_call_results": same,
        "stages_ms": {k: round(v[1] / v[0], 4) for k, v in {**prof_msm, **prof_ntt}.items()},
        "roofline": roofline,
        "roofline_alone": roofline_alone,
        "stages_live_ms": {k: round(v[1] / args.steps, 4) for k, v in prof_live.items()},
        "ntt_roofline": ntt_roof,
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "autotune": tuned,
        "batched": batched,
        "served": served,
        "int64": int64,
    }
    return line


def _profile_traffic(kernel: str, n: int) -> float | None:
    """DRAM bytes per launch of *kernel* from a committed ncu summary (profiles/*.txt lines
    `traffic <kernel> <points> <bytes>`): the capture at exactly n points, else the largest
    capture scaled to n; None when not captured yet."""
    found: dict[float, float] = {}
    for f in sorted((ROOT / "profiles").glob("*.txt")):
        for line in f.read_text().splitlines():
            parts = line.split()
            if len(parts) == 4 and parts[0] == "traffic" and parts[1] == kernel:
                try:
                    found[float(parts[2])] = float(parts[3])
                except ValueError:
                    continue
    if not found:
        return None
    if float(n) in found:
        return round(found[float(n)])
    points = max(found)
    return round(found[points] * n / points)


def release_cached_memory() -> None:
    """Return the caching allocator's free blocks to the device (between legs, untimed)."""
    import gc

    import torch

    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def _run_e2e(args, step: Step, dist, device, log_msm: int, log_ntt: int) -> dict:
    """The same step through the public API with pinned host inputs and host results.

    The timed form stages the step's inputs over PCIe on one copy stream: the
    uniform scalars with the base set (copied once, shared by both MSMs), the two
    NTT inputs, then the skewed scalars. The four public-API calls
    (msm_pippenger_affine x2, to_montgomery / ntt / from_montgomery x2) are issued
    from four host threads, each on its own stream waiting for its own inputs; the
    NTT streams have the higher priority, so each transform finishes soon after
    its input lands and its result crosses PCIe back while the MSMs compute. Two
    more forms are timed beside it: the four calls given the host tensors (each
    copies its own inputs, the bases twice) and the same calls one after another."""
    import numpy as np
    import torch

    from zkgpu import curve_gpu, msm_gpu
    from zkgpu.field256_gpu import BN254_FQ, BN254_FR

    # host inputs: plain affine coordinates, plain scalars, plain NTT input (pinned)
    plain = BN254_FQ.from_montgomery(step.bases.reshape(-1, 4)).reshape(-1, 2, 4).cpu().pin_memory()
    su = torch.from_numpy(step.sc_uniform_host).pin_memory()
    ss = torch.from_numpy(step.sc_skewed_host).pin_memory()
    xin = torch.from_numpy(step.ntt_plain_host).pin_memory()
    youts = [torch.empty_like(xin).pin_memory() for _ in range(2)]
    h2d = plain.numel() * 8 + su.numel() * 8 + ss.numel() * 8 + 2 * xin.numel() * 8
    h2d_api = h2d + plain.numel() * 8
    d2h = 2 * youts[0].numel() * 8 + 2 * 80
    results: list = [None] * 4
    # device input buffers, allocated once as a serving process would keep them
    x_dev = [torch.empty(xin.shape, dtype=xin.dtype, device=device) for _ in range(2)]
    su_dev = torch.empty(su.shape, dtype=su.dtype, device=device)
    ss_dev = torch.empty(ss.shape, dtype=ss.dtype, device=device)
    b_dev = torch.empty(plain.shape, dtype=plain.dtype, device=device)

    def part(i: int, staged: bool) -> None:
        if i < 2:
            pts = b_dev if staged else plain
            sc = (su_dev, ss_dev)[i] if staged else (su, ss)[i]
            results[i] = msm_gpu.msm_pippenger_affine(pts, sc, window_size=None)
        else:
            coset = None if i == 2 else COSET
            x = x_dev[i - 2] if staged else xin
            y = BN254_FR.from_montgomery(BN254_FR.ntt(BN254_FR.to_montgomery(x), coset=coset))
            youts[i - 2].copy_(y, non_blocking=staged)

    from concurrent.futures import ThreadPoolExecutor

    lo, hi = torch.cuda.Stream.priority_range()
    streams = [torch.cuda.Stream(device, priority=hi if i >= 2 else 0) for i in range(4)]
    copy = torch.cuda.Stream(device)
    ready = [torch.cuda.Event() for _ in range(4)]
    pool = ThreadPoolExecutor(4)
    start = torch.cuda.Event(enable_timing=True)

    def stage_inputs() -> None:
        # the longest MSM's inputs first, then both NTT inputs, the skewed scalars last:
        # each transform's 512 MB result then crosses PCIe back while the MSMs still
        # compute (measured on B200: 46.8 against 49.2 ms with the skewed scalars second)
        copy.wait_event(start)
        with torch.cuda.stream(copy):
            su_dev.copy_(su, non_blocking=True)
            b_dev.copy_(plain, non_blocking=True)
            ready[0].record(copy)
            x_dev[0].copy_(xin, non_blocking=True)
            ready[2].record(copy)
            x_dev[1].copy_(xin, non_blocking=True)
            ready[3].record(copy)
            ss_dev.copy_(ss, non_blocking=True)
            ready[1].record(copy)

    def on_stream(i: int, staged: bool) -> None:
        torch.cuda.set_device(device)
        streams[i].wait_event(ready[i] if staged else start)
        with torch.cuda.stream(streams[i]):
            part(i, staged)

    def e2e_step(staged: bool = True) -> None:
        if staged:
            stage_inputs()
        for f in [pool.submit(on_stream, i, staged) for i in (0, 1, 2, 3)]:
            f.result()

    def sequential_step() -> None:
        for i in range(4):
            part(i, False)

    steps = max(2, min(args.steps, 5))
    main = torch.cuda.current_stream()

    def once(fn) -> None:
        start.record(main)  # this step's streams start after everything before it
        fn()
        for s in streams + [copy]:
            main.wait_stream(s)

    def timed(fn) -> float:
        begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        begin.record(main)
        for _ in range(steps):
            once(fn)
        end.record(main)
        torch.cuda.synchronize()
        return begin.elapsed_time(end) / steps

    for _ in range(max(1, args.warmup)):
        for fn in (lambda: e2e_step(True), lambda: e2e_step(False), sequential_step):
            once(fn)
    torch.cuda.synchronize()
    barrier(dist, device)
    t0 = time.perf_counter()
    ms = max_over_ranks(timed(lambda: e2e_step(True)), dist, device)
    wall = (time.perf_counter() - t0) * 1e3 / steps
    ref = [results[0], results[1], youts[0].clone(), youts[1].clone()]
    api_ms = max_over_ranks(timed(lambda: e2e_step(False)), dist, device)
    same = results[:2] == ref[:2] and all(bool(torch.equal(y, r)) for y, r in zip(youts, ref[2:]))
    seq = max_over_ranks(timed(sequential_step), dist, device)
    pool.shutdown()
    return {"value": round(ms, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "steps": steps, "wall_ms": round(wall, 3),
            "api_copies_ms": round(api_ms, 3), "api_copies_h2d_bytes_per_step": int(h2d_api),
            "sequential_ms": round(seq, 3), "same_results": same,
            "api": "zkgpu.msm_gpu.msm_pippenger_affine x2, Field256.to_montgomery/ntt/from_montgomery x2 from four "
                   "host threads on four streams, inputs staged on one copy stream: the uniform MSM's inputs (the "
                   "base set copied once), the NTT inputs, the skewed scalars; NTTs on high-priority streams; "
                   "api_copies_ms: the same calls "
                   "given the host tensors (each copies its own inputs); sequential_ms: one after another"}


def full_size_parity(step: Step, plan_outs: list, digest: str) -> dict:
    """The timed step's four results against the C port of the reference's CPU algorithms
    at full size (all host threads): bit for bit, and by the same SHA-256 the reference
    arm prints."""
    import numpy as np

    threads = os.cpu_count() or 1
    bases_h = step.bases.cpu().numpy()
    ntt_h = step.ntt_in.cpu().numpy()
    outs, secs = oracle_outputs(bases_h, step.sc_uniform_host, step.sc_skewed_host, ntt_h, threads)
    same = [bool(np.array_equal(np.asarray(a, dtype=np.uint64).reshape(-1)[:9], b.reshape(-1)[:9]))
            for a, b in zip(outs[:2], plan_outs[:2])]
    same += [bool(np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64)))
             for a, b in zip(outs[2:], plan_outs[2:])]
    oracle_digest = outputs_sha256(*outs)
    return {"same": all(same) and oracle_digest == digest,
            "parts": dict(zip(("msm_uniform", "msm_skewed", "ntt", "coset_ntt"), same)),
            "oracle_sha256": oracle_digest, "oracle_s": round(secs, 2), "threads": threads,
            "oracle": "C port of the reference's CPU Pippenger and Radix-2 NTT (oracle/zk_oracle.c), full size"}


def run_sharded(args, step: Step, dist, device, rank: int, world: int, log_msm: int, log_ntt: int) -> dict:
    """Strong scaling beside the replicas: ONE 2^log_msm uniform MSM with its points split
    over the ranks (each rank's partial sum, one all-gather of 72-byte results) and ONE
    2^log_ntt NTT split four-step over the ranks (two all-to-all exchanges, cyclic output),
    both over NCCL (zkgpu.sharded). Device time per operation with CUDA events, max over
    ranks. Rank 0's results are checked against its own one-GPU results of the same
    inputs (rank 0's replica uses the same seeds)."""
    import numpy as np
    import torch

    from zkgpu import curve_gpu, sharded, workloads as wl
    from zkgpu.field256_gpu import BN254_FR

    n, m = 1 << log_msm, 1 << log_ntt
    lo, hi = sharded.shard_bounds(n, world, rank)
    pts = curve_gpu.mul_generator(wl.base_scalars(10, n)[lo:hi])
    sc = torch.from_numpy(np.ascontiguousarray(wl.uniform_fr(11, n)[lo:hi])).to(device)
    mlo, mhi = sharded.shard_bounds(m, world, rank)
    x = BN254_FR.to_montgomery(np.ascontiguousarray(wl.uniform_fr(13, m)[mlo:mhi]))
    torch.cuda.synchronize()
    reps = 3

    def timed(fn) -> tuple[float, object]:
        out = None
        for _ in range(2):
            out = fn()
        torch.cuda.synchronize()
        barrier(dist, device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            out = fn()
        b.record()
        torch.cuda.synchronize()
        return max_over_ranks(a.elapsed_time(b) / reps, dist, device), out

    msm_ms, point = timed(lambda: sharded.msm_sharded(pts, sc, window_size=step.w))
    ntt_ms, y = timed(lambda: sharded.ntt_sharded(x))
    checks = None
    if rank == 0:
        from zkgpu.batch import results_to_points

        one_gpu = results_to_points(step.plan.msm_results[:1])[0]
        want = step.plan.ntt_outputs[0][0::world]  # rank 0's cyclic slice: y[0], y[G], ...
        checks = {"msm_same_as_one_gpu": point == one_gpu, "ntt_slice_same_as_one_gpu": bool(torch.equal(y, want))}
    return {"scaling": "strong", "ranks": world, "msm_ms": round(msm_ms, 3), "ntt_ms": round(ntt_ms, 3),
            "msm": f"one 2^{log_msm} uniform MSM, {n // world}-point slices, one all-gather",
            "ntt": f"one 2^{log_ntt} NTT, four-step over {world} ranks, two all-to-all exchanges (cyclic output)",
            "timing": f"CUDA events, mean of {reps} after 2 warm-up, max over ranks", "checks": checks}


# ------------------------------------------------------------------
# Batched form (64 NTTs + 32 MSMs) and served form (Poisson stream of prover jobs)
# ------------------------------------------------------------------


def _event_ms(fn, reps: int) -> float:
    import torch

    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def run_batched(seed: int = 6, log_base: int = 20, table_windows: tuple[int, ...] = (15, 16, 17)) -> dict:
    """64 Fr NTTs (sizes 2^U{10..20}, uniform inputs) + 32 G1 MSMs (sizes 2^U(12, 20) over
    prefixes of one resident 2^20 base set, uniform scalars): one-at-a-time calls (zkb_ntt and
    zkb_msm per job, the drop-in path) against one BatchPlan run (one persistent NTT launch + one
    MSM batch) and its CUDA-graph replay.

    The batch is tuned for its shape: the MSM jobs share the resident base set, so the batch
    runs them over a fixed-base table of it, and the table's window is chosen by timing the
    whole batch at each candidate window (`autotune`); the variable-base batch, with the
    library's per-size windows, is timed beside it, and so is one call per job over the chosen
    table, so the ratio of every form is on the line."""
    import ctypes

    import numpy as np
    import torch

    from zkgpu import _native, batch, curve_gpu, workloads as wl
    from zkgpu.field256_gpu import BN254_FR
    from zkgpu.msm_gpu import FixedBaseTable

    rng = np.random.default_rng(seed)
    ntt_sizes = [1 << int(v) for v in rng.integers(10, log_base + 1, size=64)]
    msm_sizes = [int(2 ** v) for v in rng.uniform(12, log_base, size=32)]
    bases = curve_gpu.mul_generator(wl.base_scalars(seed, 1 << log_base))
    xs = [BN254_FR.to_montgomery(wl.uniform_fr(1000 + k, n)) for k, n in enumerate(ntt_sizes)]
    scs = [torch.from_numpy(wl.uniform_fr(2000 + k, n)).cuda() for k, n in enumerate(msm_sizes)]
    lib = _native.lib()
    f = BN254_FR._field()
    outs = [torch.empty_like(x) for x in xs]
    ntt_ws = [_native.workspace(lib.zkb_ntt_workspace_bytes(n)) for n in ntt_sizes]
    msm_ws = [_native.workspace(lib.zkb_msm_workspace_bytes(n, 0)) for n in msm_sizes]
    res = torch.empty((32, 16), dtype=torch.int64, device="cuda")

    def plain() -> None:
        s = _native.stream_ptr()
        for k, n in enumerate(ntt_sizes):
            _native.check(lib.zkb_ntt(ctypes.byref(f), xs[k].data_ptr(), outs[k].data_ptr(), n, 0, None, None,
                                      ntt_ws[k].data_ptr(), ntt_ws[k].numel(), s))
        for k, n in enumerate(msm_sizes):
            _native.check(lib.zkb_msm(bases.data_ptr(), scs[k].data_ptr(), n, 0, res[k].data_ptr(),
                                      msm_ws[k].data_ptr(), msm_ws[k].numel(), s))

    t_plain = _event_ms(plain, 3)
    ntt_jobs = [(x, False, None) for x in xs]
    msm_jobs = [(bases[:n], scs[k], None) for k, n in enumerate(msm_sizes)]

    def check(plan) -> bool:
        return all(bool((o == y).all()) for o, y in zip(outs, plan.ntt_outputs)) and \
            bool((res[:, :9] == plan.msm_results[:32, :9]).all())

    # the variable-base batch (per-size windows, one pipeline per window group)
    vplan = batch.BatchPlan(ntt_jobs=ntt_jobs, msm_jobs=msm_jobs)
    t_var = _event_ms(vplan.run, 3)
    same = check(vplan)
    del vplan
    # the table window, tuned for this batch by timing it
    tuned: dict[int, float] = {}
    build_ms: dict[int, float] = {}
    best = None
    for w in table_windows:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        table = FixedBaseTable(bases, w)
        torch.cuda.synchronize()
        build_ms[w] = (time.perf_counter() - t0) * 1e3
        plan = batch.BatchPlan(ntt_jobs=ntt_jobs, msm_jobs=msm_jobs, table=table)
        tuned[w] = _event_ms(plan.run, 3)
        same = same and check(plan)
        if best is None or tuned[w] < tuned[best[0]]:
            best = (w, table, plan)
        else:
            del plan, table
    w_best, table, plan = best
    t_batch = tuned[w_best]
    plan.capture()
    t_graph = _event_ms(plan.replay, 3)
    plan.check_status()
    same = same and check(plan)
    # one call per job over the same table (the batch's MSM algorithm without the batching)
    single = []
    for k, n in enumerate(msm_sizes):
        j = (_native.ZkbMsmJob * 1)()
        j[0].points, j[0].scalars, j[0].n = _native.ptr(table.table), scs[k].data_ptr(), n
        j[0].result, j[0].window_size = res[k].data_ptr(), w_best
        single.append((j, _native.workspace(lib.zkb_msm_fixed_batch_workspace_bytes(j, 1))))

    def plain_table() -> None:
        s = _native.stream_ptr()
        for k, n in enumerate(ntt_sizes):
            _native.check(lib.zkb_ntt(ctypes.byref(f), xs[k].data_ptr(), outs[k].data_ptr(), n, 0, None, None,
                                      ntt_ws[k].data_ptr(), ntt_ws[k].numel(), s))
        for j, ws in single:
            _native.check(lib.zkb_msm_fixed_batch(j, 1, ws.data_ptr(), ws.numel(), s))

    t_plain_table = _event_ms(plain_table, 3)
    jobs = len(ntt_sizes) + len(msm_sizes)
    best_ms = min(t_batch, t_graph)
    return {
        "workload": f"64 Fr NTTs 2^U{{10..{log_base}}} + 32 G1 MSMs 2^U(12,{log_base}) over one resident "
                    f"2^{log_base} base set (seed {seed})",
        "jobs": jobs, "plain_ms": round(t_plain, 3), "batched_ms": round(t_batch, 3), "graph_ms": round(t_graph, 3),
        "plain_jobs_per_s": round(jobs / t_plain * 1e3, 1), "batched_jobs_per_s": round(jobs / t_batch * 1e3, 1),
        "graph_jobs_per_s": round(jobs / t_graph * 1e3, 1), "speedup": round(t_plain / best_ms, 3),
        "plain": "one zkb_ntt / zkb_msm call per job (the drop-in path, variable-base MSMs)",
        "batched": f"one NTT batch launch + one MSM batch over a fixed-base table of the resident base set "
                   f"(w = {w_best}, {table.nbytes >> 20} MiB, built once in {build_ms[w_best]:.0f} ms)",
        "variable_base_batched_ms": round(t_var, 3), "variable_base_speedup": round(t_plain / t_var, 3),
        "plain_over_table_ms": round(t_plain_table, 3),
        "speedup_same_msm_algorithm": round(t_plain_table / best_ms, 3),
        "autotune": {"table_window_ms": {str(k): round(v, 3) for k, v in tuned.items()}, "chosen": w_best,
                     "how": "the whole batch timed at each candidate table window (CUDA events, mean of 3)"},
        "launches_per_batch": plan.launches_per_run, "same_results": same,
        "timing": "CUDA events, mean of 3 after 2 warm-up",
    }


INT64_NTT_PRIME = 2_147_483_641 * 2**32 + 1  # largest prime below 2^63 of the form k 2^32 + 1


def run_int64(log_n: int = 25, log_ops: int = 26, cpu: bool = True) -> dict:
    """The int64 field path (moduli below 2^63): one forward NTT of 2^log_n words over
    INT64_NTT_PRIME and one element-wise product of 2^log_ops words, both larger than L2,
    each timed with CUDA events through the C ABI; the oracle's NumPy NTT of 2^20 words
    over 998244353 on one host thread beside them."""
    import ctypes

    import torch

    from zkgpu import _native, field_gpu
    from zkgpu.ntt_gpu import ntt_gpu
    from zkgpu.roots import get_ntt_root

    lib, peaks = _native.lib(), _peaks()
    n = 1 << log_n
    g = torch.Generator(device="cuda").manual_seed(64)
    x = torch.randint(0, INT64_NTT_PRIME, (n,), device="cuda", generator=g)
    y = torch.empty_like(x)
    omega = get_ntt_root(n, INT64_NTT_PRIME)
    ws_bytes = int(lib.zkb_ntt64_workspace_bytes(n))
    ws = _native.workspace(ws_bytes)

    def ntt() -> None:
        _native.check(lib.zkb_ntt64(x.data_ptr(), y.data_ptr(), n, INT64_NTT_PRIME, omega, 0, ws.data_ptr(),
                                    ctypes.c_size_t(ws_bytes), _native.stream_ptr()))

    t_ntt = _event_ms(ntt, 10)
    same = bool(torch.equal(ntt_gpu(y, INT64_NTT_PRIME, invert=True), x))
    m = 1 << log_ops
    a = torch.randint(0, INT64_NTT_PRIME, (m,), device="cuda", generator=g)  # field elements, as the
    b = torch.randint(0, INT64_NTT_PRIME, (m,), device="cuda", generator=g)  # reference's tests draw them
    c = torch.empty_like(a)

    def mul() -> None:
        _native.check(lib.zkb_u64_mul(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, INT64_NTT_PRIME,
                                      _native.stream_ptr()))

    t_mul = _event_ms(mul, 10)
    same = same and bool(torch.equal(c[:1024], field_gpu.gpu_batch_mul(a[:1024], b[:1024], INT64_NTT_PRIME)))
    hbm = peaks.get("hbm_gbs") or 6650.0  # else the earlier measurement on this pool
    ntt_gbs = 16 * n / t_ntt / 1e6
    mul_gbs = 24 * m / t_mul / 1e6
    passes = 1 + -(-(log_n - 10) // 10)
    # a modulus below 2^31 (998244353 = 119 2^23 + 1, its largest size): the 32-bit butterflies
    small = torch.randint(0, 998_244_353, (1 << 23,), device="cuda", generator=g)
    t_small = _event_ms(lambda: ntt_gpu(small, 998_244_353), 10)
    out = {
        "workload": f"forward NTT of 2^{log_n} int64 words mod {INT64_NTT_PRIME} (k 2^32 + 1); "
                    f"element-wise product of 2^{log_ops} words",
        "ntt_998244353_2e23_ms": round(t_small, 4),
        "ntt_ms": round(t_ntt, 4),
        "ntt_passes": passes,
        "ntt_roofline": {"bound": "hbm", "achieved": round(ntt_gbs, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(ntt_gbs / hbm, 3),
                         "algorithmic_bytes": f"16 B/word (one read, one write) x 2^{log_n}; the kernel makes "
                                              f"{passes} passes over HBM"},
        "mul_ms": round(t_mul, 4),
        "mul_roofline": {"bound": "hbm", "achieved": round(mul_gbs, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(mul_gbs / hbm, 3), "algorithmic_bytes": "24 B/word (two reads, one write)",
                         "inputs": "uniform in [0, mod)"},
        "same_results": same,
        "timing": "CUDA events on the launching stream, mean of 10 after 2 warm-up; inputs larger than L2",
    }
    if cpu:
        import numpy as np

        from oracle import pyoracle as po

        v = np.random.default_rng(20).integers(0, 998_244_353, 1 << 20)
        t0 = time.perf_counter()
        po.ntt_np(v, 998_244_353)
        cpu_ms = (time.perf_counter() - t0) * 1e3
        z = torch.from_numpy(v).cuda()
        gpu_ms = _event_ms(lambda: ntt_gpu(z, 998_244_353), 10)
        out["cpu_baseline"] = {"value": round(cpu_ms, 2), "unit": "ms per 2^20-word NTT mod 998244353",
                               "cores": 1, "kind": "port",
                               "sample": "the oracle's NumPy NTT (stage-vectorised, as the reference's ntt_gpu "
                                         "runs its stages); the reference's own CPU fallback is the pure-Python "
                                         "NTT, slower still",
                               "gpu_ms_same_case": round(gpu_ms, 4)}
    return out


def run_served(n_jobs: int = 2000, rate: float = 200.0, log_max: int = 20, seed: int = 7, runs: int = 3,
               table_window: int = 16) -> dict:
    """Poisson stream (rate jobs/s) of Groth16-shaped jobs, m = 2^U{12..log_max}: each job 3
    inverse NTTs, 3 coset NTTs, the pointwise quotient, 1 inverse coset NTT and 4 G1 MSMs
    (skewed witness scalars; h for the last) over a resident base set. The served form
    (zkgpu.serving) against the same jobs one at a time (prove_plain, a 60-job sample). The
    base set stays resident, as a prover's SRS does, so both forms run their MSMs over one
    fixed-base table of it (table_window; 0 = the plain MSM), built once before either runs."""
    import numpy as np
    import torch

    from zkgpu import curve_gpu, workloads as wl
    from zkgpu.msm_gpu import FixedBaseTable
    from zkgpu.prover import ProofJob, prove_plain, synthetic_request
    from zkgpu.serving import Server, summarize

    bases = curve_gpu.mul_generator(wl.base_scalars(seed, 1 << log_max))
    torch.cuda.synchronize()
    t_build = time.perf_counter()
    table = FixedBaseTable(bases, table_window) if table_window else None
    torch.cuda.synchronize()
    t_build = (time.perf_counter() - t_build) * 1e3
    pool = {1 << e: [synthetic_request(1000 * e + k, 1 << e) for k in range(2)] for e in range(12, log_max + 1)}
    rng = np.random.default_rng(seed)
    exps = rng.integers(12, log_max + 1, size=n_jobs)
    reqs = [pool[1 << int(e)][k % 2] for k, e in enumerate(exps)]
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_jobs))
    for group in pool.values():
        for q in group:
            q.host_rows()
    sample = reqs[: min(60, n_jobs)]
    ws: dict = {}
    # warm-up: one job of every size in the sample, so the timed loop below meets no new
    # buffer size (the allocator would otherwise grow inside it, at cudaMalloc's cost)
    for r in {q.m: q for q in sample}.values():
        prove_plain(ProofJob(r, bases), ws, table)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in sample:
        prove_plain(ProofJob(r, bases), ws, table)
        torch.cuda.synchronize()
    plain_s = time.perf_counter() - t0
    budget = 60 << 30
    # warm-up: the first 200 jobs queued at once, untimed. It builds the tables and grows the
    # allocator's pool (on the servers' streams, which every Server shares) to the largest
    # number of jobs in flight, so no timed run below stops for device allocations.
    n_cap = min(200, n_jobs)
    Server(bases, budget, table=table).run(reqs[:n_cap], [0.0] * n_cap)
    # capacity: the same 200 jobs queued at once (closed loop), twice; the mean of the two
    cap_rates = []
    for _ in range(2):
        cap = Server(bases, budget, table=table)
        t0 = time.perf_counter()
        cap_recs = cap.run(reqs[:n_cap], [0.0] * n_cap)
        cap_rates.append(summarize(cap_recs, time.perf_counter() - t0)["jobs_per_s"])
    cap_s = {"jobs_per_s": sum(cap_rates) / len(cap_rates)}
    # the same Poisson stream served `runs` times: the line's latencies are the median run's,
    # with every run's p50 / p99 beside them for the run-to-run spread
    summaries = []
    for _ in range(runs):
        srv = Server(bases, budget, table=table)
        t0 = time.perf_counter()
        recs = srv.run(reqs, list(arrivals))
        summaries.append(summarize(recs, time.perf_counter() - t0))
    by_p99 = sorted(range(runs), key=lambda k: summaries[k]["p99_ms"])
    s = summaries[by_p99[runs // 2]]
    p99s = [round(x["p99_ms"], 2) for x in summaries]
    plain_jobs_s = len(sample) / plain_s
    return {
        "workload": f"{n_jobs} Groth16-shaped jobs, Poisson {rate:g}/s, m = 2^U{{12..{log_max}}}, 7 NTTs + "
                    f"4 G1 MSMs each, resident 2^{log_max} base set (seed {seed})",
        "jobs": n_jobs, "rate_per_s": rate, "jobs_per_s": round(s["jobs_per_s"], 1),
        "p50_ms": round(s["p50_ms"], 2), "p90_ms": round(s["p90_ms"], 2), "p99_ms": round(s["p99_ms"], 2),
        "max_ms": round(s["max_ms"], 2),
        "runs": runs, "p50_ms_runs": [round(x["p50_ms"], 2) for x in summaries], "p99_ms_runs": p99s,
        "p99_spread": round(max(p99s) / max(min(p99s), 1e-9), 3),
        "plain_jobs_per_s": round(plain_jobs_s, 1),
        "speedup_vs_plain": round(s["jobs_per_s"] / plain_jobs_s, 3),
        "capacity_jobs_per_s": round(cap_s["jobs_per_s"], 1),
        "capacity_runs_jobs_per_s": [round(x, 1) for x in cap_rates],
        "capacity_vs_plain": round(cap_s["jobs_per_s"] / plain_jobs_s, 3),
        "capacity": "the first 200 jobs queued at once (closed loop): the mean of two runs after one untimed run",
        "plain": f"the first {len(sample)} jobs one at a time (one call per NTT / MSM, synchronised per job)",
        "ticks": srv.ticks, "gpu_launches": srv.launches, "hbm_budget_bytes": budget,
        "latency": "arrival (host clock) to the device-side completion of the job's last MSM batch",
        "msm": (f"over a fixed-base table of the resident base set (w = {table_window}, "
                f"{table.nbytes >> 20} MiB, built once in {t_build:.0f} ms), served and plain alike")
               if table is not None else "zkb_msm_batch / zkb_msm over the base set",
    }


# ------------------------------------------------------------------
# CPU baseline: the oracle (C port of the reference's CPU algorithms)
# ------------------------------------------------------------------


def _timed(fn) -> float:
    t0 = time.perf_counter()
    fn()
    return time.perf_counter() - t0


def cpu_estimate(bases_h, sc_u, sc_s, ntt_h, log_ntt: int, threads: int, full: bool) -> tuple[float, str]:
    """Estimated ms of one step of the reference's CPU algorithms (the C oracle).

    MSM at the reference's window for n (w = 16 at 2^22, zkgpu/msm.py:112-121):
    windows are timed individually at full n and summed as w0 + w1 + (W - 2) w2
    (windows 2.. hold the same digit statistics; w0/w1 carry the small scalars).
    NTT: the bit-reversal copy plus a sample of butterfly stages (each stage is
    n/2 butterflies), scaled to all log2 n stages; coset adds its scaling pass.
    With full=True every window and stage runs (no scaling).
    """
    from oracle import c_oracle as co
    from oracle import pyoracle as po

    n = bases_h.shape[0]
    w = po.pippenger_window_size(n)
    W = -(-SCALAR_BITS // w)
    total = 0.0
    notes = []
    for name, sc in (("uniform", sc_u), ("skewed", sc_s)):
        if full:
            t = _timed(lambda sc=sc: co.msm(bases_h, sc, w, threads=threads))
        else:
            t0 = _timed(lambda sc=sc: co.msm_window_sums(bases_h, sc, w, 0, 1, threads=1))
            t1 = _timed(lambda sc=sc: co.msm_window_sums(bases_h, sc, w, 1, 2, threads=1))
            t2 = _timed(lambda sc=sc: co.msm_window_sums(bases_h, sc, w, 2, 3, threads=1))
            t = t0 + t1 + (W - 2) * t2
        total += t
        notes.append(f"msm {name} 2^{n.bit_length() - 1} w={w}: {t * 1e3:.0f} ms")
    m = ntt_h.shape[0]
    if full:
        t_ntt = _timed(lambda: co.ntt(ntt_h, threads=threads))
        t_coset = _timed(lambda: co.ntt(ntt_h, coset=COSET, threads=threads))
    else:
        sample = 2
        t_rev = _timed(lambda: co.ntt(ntt_h, threads=threads, stages=(0, 0)))
        t_st = (_timed(lambda: co.ntt(ntt_h, threads=threads, stages=(0, sample))) - t_rev) / sample
        t_scale = _timed(lambda: co.ntt(ntt_h, coset=COSET, threads=threads, stages=(0, 0))) - t_rev
        t_ntt = t_rev + log_ntt * t_st
        t_coset = t_ntt + max(t_scale, 0.0)
    total += t_ntt + t_coset
    notes.append(f"ntt 2^{log_ntt}: {t_ntt * 1e3:.0f} ms, coset: {t_coset * 1e3:.0f} ms")
    return total * 1e3, "; ".join(notes)


def cpu_baseline_sample(step: Step, threads: int) -> dict:
    from oracle import c_oracle as co

    bases_h = step.bases.cpu().numpy()
    ntt_h = step.ntt_in.cpu().numpy()
    log_ntt = step.m.bit_length() - 1
    ms, notes = cpu_estimate(bases_h, step.sc_uniform_host, step.sc_skewed_host, ntt_h, log_ntt, threads, False)
    return {"value": round(ms, 1), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "C port of the reference's CPU algorithms (oracle/zk_oracle.c) on the same inputs: "
                      "MSM windows 0, 1, 2 at full n scaled to all windows; NTT bit reversal + 2 of "
                      f"{log_ntt} stages scaled; " + notes,
            "host_cpus": os.cpu_count()}


# ------------------------------------------------------------------
# Reference arm
# ------------------------------------------------------------------


def oracle_outputs(bases_h, sc_u, sc_s, ntt_h, threads: int) -> tuple[list, float]:
    """The step's four results from the C port of the reference's CPU algorithms, and the
    seconds it took: MSMs at the reference's window for n (zkgpu/msm.py:112-121), the NTT and
    the coset NTT (zkgpu/ntt.py:149-203, zkgpu/domain.py:122-135) on Montgomery rows."""
    from oracle import c_oracle as co
    from oracle import pyoracle as po

    w = po.pippenger_window_size(bases_h.shape[0])
    t0 = time.perf_counter()
    outs = [co.msm(bases_h, sc_u, w, threads=threads), co.msm(bases_h, sc_s, w, threads=threads),
            co.ntt(ntt_h, threads=threads), co.ntt(ntt_h, coset=COSET, threads=threads)]
    return outs, time.perf_counter() - t0


def run_reference(args, rank: int, world: int) -> dict | None:
    """The reference's CPU algorithms (C port, all host threads) on the same workload.

    One untimed full step first (its outputs give `outputs_sha256`, comparable with the
    GPU arm's), then exactly --steps timed steps: the whole step when --steps of them fit
    in about 150 s at the full step's speed, else each step the bounded sample of
    cpu_estimate (MSM windows 0-2 at full n, 2 NTT stages, scaled). Rank 0 alone runs."""
    if rank != 0:
        return None
    from oracle import c_oracle as co
    from zkgpu import workloads as wl

    log_msm, log_ntt = WORKLOADS[args.workload]
    n, m = 1 << log_msm, 1 << log_ntt
    threads = os.cpu_count() or 1
    k = wl.base_scalars(10, n)
    bases_h = co.mul_generator(k, threads=threads)
    sc_u, sc_s = wl.uniform_fr(11, n), wl.skewed_scalars(12, n)
    ntt_h = co.to_mont(co.FR, wl.uniform_fr(13, m))
    outs, full_s = oracle_outputs(bases_h, sc_u, sc_s, ntt_h, threads)
    digest = outputs_sha256(*outs)
    steps = max(1, args.steps)
    full = full_s * steps <= 150.0
    for _ in range(max(0, args.warmup - 1)):  # the full step above was the first warm-up
        cpu_estimate(bases_h, sc_u, sc_s, ntt_h, log_ntt, threads, full)
    times = []
    notes = ""
    for _ in range(steps):
        ms, notes = cpu_estimate(bases_h, sc_u, sc_s, ntt_h, log_ntt, threads, full)
        times.append(ms)
    value = statistics.mean(times)
    sample = ("full step" if full else "bounded sample (MSM windows 0-2 at full n, NTT 2 of "
              f"{log_ntt} stages, scaled; the full step took {full_s:.1f} s)") + \
        f" with {threads} threads, mean of {steps} timed steps; " + notes
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": args.warmup, "steps_timed": steps, "ms_per_step": round(value, 1),
        "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (4x64-bit limb Montgomery, exact)",
        "data": "synthetic (seeded)",
        "config": workload_config(log_msm, log_ntt, world),
        "outputs_sha256": digest,
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[1])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="large")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    ap.add_argument("--skip-batched", action="store_true", help="skip the batched form (64 NTTs + 32 MSMs)")
    ap.add_argument("--skip-served", action="store_true", help="skip the served form (Poisson job stream)")
    ap.add_argument("--skip-int64", action="store_true", help="skip the int64 field / NTT figures")
    ap.add_argument("--knob", action="append", default=[], metavar="KEY=VALUE",
                    help="set a library tuning knob (zkb_tune_set) before the run; repeatable")
    ap.add_argument("--tune", action="store_true",
                    help="measure (or load from the cache) per-size MSM windows and NTT shapes first")
    ap.add_argument("--skip-parity", action="store_true",
                    help="skip the full-size bit-exact check of the timed outputs against the C oracle")
    ap.add_argument("--check-ranks", action="store_true",
                    help="run only the multi-rank plumbing (spawn, process group, barrier, max over ranks)")
    args = ap.parse_args()
    if args.gpus < 1:
        ap.error("--gpus must be at least 1")
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # no launcher: start one rank per GPU here (torchrun sets WORLD_SIZE itself)
        sys.exit(spawn_ranks(args.gpus, sys.argv[1:]))
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3  # at least three untimed steps
    rank, world, local_rank = dist_env()
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but the launcher started {world} ranks")
    if args.check_ranks:
        line = check_ranks(args, rank, world, local_rank)
    elif args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local_rank)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
