"""
zkgpu.serving — a continuous-batching service for Groth16-shaped prover jobs.

Requests arrive over time (e.g. a Poisson stream); each is one prover job
(zkgpu.prover: 7 NTTs of size m and 4 G1 MSMs against a resident base set).
The service

- admits queued jobs first-come first-served while the device memory of the
  jobs in flight stays within an HBM budget (a job larger than the whole
  budget runs alone);
- advances every job in flight by one stage per tick, and launches each
  tick's work for ALL jobs together: the tick's transforms of every job in
  one persistent NTT launch (zkb_ntt_batch, 64 per launch), the fused
  quotient steps;
- queues the MSMs: the A, B and L MSMs of a job when it is admitted (they
  need only the witness), its H MSM when h is ready. Each of two
  high-priority MSM streams takes the queued MSMs, first come first served
  up to 2^22 points, as one batch (zkb_msm_batch) whenever its previous
  batch has finished: batches grow with the load and share one sort, bucket
  pass and tail; one batch's latency-bound tail overlaps the other stream's
  accumulation; the ticks' transforms fill the SMs the MSMs leave idle.
  (Measured at 200 jobs/s: high-priority MSMs with the 2^22 cap gave p99
  159 ms; the reverse priorities, larger caps or taking the whole queue,
  0.6-1.4 s);
- admits new jobs at every tick, while others are on the GPU: continuous
  batching, not a queue in front of one-at-a-time launches;
- reports each job's latency (arrival to the device-side completion of its
  last MSM) and the throughput.

Stages (one per tick): INTT (host rows copied on a stream of their own,
while the tick's other transforms and the MSM batches run; 3 inverse NTTs;
A, B, L MSMs start once the witness is on the device) -> COSET (3 coset NTTs)
-> QUOTIENT (pointwise + inverse coset NTT + h to plain form) -> MSM (the H
MSM) -> done when both MSM batches completed.

Scheduler holds the policy and needs no GPU (tested on the CPU with a fake
clock); Server drives it on the device.
"""

from __future__ import annotations

import ctypes
import time
from collections import deque
from collections.abc import Callable, Sequence
from dataclasses import dataclass, field
from typing import Any

from zkgpu import _native
from zkgpu.prover import (
    COSET,
    STAGE_COSET,
    STAGE_DONE,
    STAGE_INTT,
    STAGE_MSM,
    STAGE_QUOTIENT,
    ProofJob,
    ProofRequest,
    msm_table_jobs,
)

MAX_NTT_PER_LAUNCH = 64


@dataclass
class Tick:
    """The work of one tick: job ids per stage they run in it."""

    admitted: list[int] = field(default_factory=list)
    intt: list[int] = field(default_factory=list)
    coset: list[int] = field(default_factory=list)
    quotient: list[int] = field(default_factory=list)
    msm: list[int] = field(default_factory=list)

    def empty(self) -> bool:
        return not (self.intt or self.coset or self.quotient or self.msm)


class Scheduler:
    """
    Admission and stage bookkeeping, independent of the device.

    submit(job_id, footprint, arrival) queues a job; admit(now) moves queued
    jobs that have arrived into flight while the budget allows; next_tick()
    returns the tick's work and advances every job in flight by one stage;
    finish(job_id) releases a job whose MSMs completed.
    """

    def __init__(self, hbm_budget: int, max_in_flight: int = 64) -> None:
        if hbm_budget <= 0:
            raise ValueError("the HBM budget must be positive")
        self.budget = hbm_budget
        self.max_in_flight = max_in_flight
        self.queue: deque[tuple[int, int, float]] = deque()  # (id, footprint, arrival)
        self.stage: dict[int, int] = {}
        self.footprint: dict[int, int] = {}
        self.used = 0
        self.finished: list[int] = []

    def submit(self, job_id: int, footprint: int, arrival: float) -> None:
        if self.queue and arrival < self.queue[-1][2]:
            raise ValueError("jobs must be submitted in arrival order")
        self.queue.append((job_id, footprint, arrival))

    def admit(self, now: float) -> list[int]:
        out = []
        while self.queue and self.queue[0][2] <= now and len(self.stage) < self.max_in_flight:
            job_id, fp, _ = self.queue[0]
            if self.used + fp > self.budget and self.stage:
                break  # first come, first served: later jobs wait too
            self.queue.popleft()
            self.stage[job_id] = STAGE_INTT
            self.footprint[job_id] = fp
            self.used += fp
            out.append(job_id)
        return out

    def next_tick(self, admitted: Sequence[int] = ()) -> Tick:
        t = Tick(admitted=list(admitted))
        for job_id, st in sorted(self.stage.items()):
            if st == STAGE_INTT:
                t.intt.append(job_id)
            elif st == STAGE_COSET:
                t.coset.append(job_id)
            elif st == STAGE_QUOTIENT:
                t.quotient.append(job_id)
            elif st == STAGE_MSM:
                t.msm.append(job_id)
        for job_id in t.intt + t.coset + t.quotient + t.msm:
            self.stage[job_id] += 1  # MSM -> DONE: waits for finish()
        return t

    def finish(self, job_id: int) -> None:
        if self.stage.get(job_id) != STAGE_DONE:
            raise ValueError(f"job {job_id} has not run its MSMs yet")
        del self.stage[job_id]
        self.used -= self.footprint.pop(job_id)
        self.finished.append(job_id)

    def idle(self) -> bool:
        return not self.queue and not self.stage

    def waiting_for_device(self) -> bool:
        """Every job in flight has launched all its work."""
        return bool(self.stage) and all(s == STAGE_DONE for s in self.stage.values())


@dataclass
class JobRecord:
    job_id: int
    m: int
    arrival_s: float
    admitted_s: float = 0.0
    finished_s: float = 0.0

    @property
    def latency_ms(self) -> float:
        return (self.finished_s - self.arrival_s) * 1e3


def percentile(values: Sequence[float], q: float) -> float:
    """The q-th percentile (0..100) by linear interpolation between order statistics."""
    v = sorted(values)
    if not v:
        return float("nan")
    pos = (len(v) - 1) * q / 100.0
    lo = int(pos)
    hi = min(lo + 1, len(v) - 1)
    return v[lo] + (v[hi] - v[lo]) * (pos - lo)


class Server:
    """
    Runs jobs through Scheduler on the current device.

    bases       : (N, 2, 4) Montgomery affine rows, resident (the SRS stand-in)
    hbm_budget  : device bytes the jobs in flight may hold (buffers + workspaces)
    max_ticks_ahead : ticks queued on the device before the host waits
    max_batch_points : an MSM stream takes queued MSMs first come, first served
                  up to this many points per batch (a bigger group still goes alone)
    msm_priority / tick_priority : "high", "normal" or "low" stream priority of
                  the MSM batches and of the ticks' transforms (the block
                  scheduler serves waiting blocks of higher-priority streams
                  first)
    table       : optional FixedBaseTable built from `bases`: the MSM batches then
                  run over it (zkb_msm_fixed_batch), with the same results
    max_in_flight : jobs admitted at once at most (the HBM budget may admit fewer)
    """

    def __init__(self, bases: Any, hbm_budget: int, max_ticks_ahead: int = 2, msm_streams: int = 2,
                 msm_priority: str = "high", tick_priority: str = "normal",
                 max_batch_points: int = 1 << 22, table: Any = None, max_in_flight: int = 256) -> None:
        torch = _native.require_cuda()
        self.torch = torch
        self.bases = bases
        self.table = table
        self.sched = Scheduler(hbm_budget, max_in_flight)
        self.max_ticks_ahead = max_ticks_ahead
        lo, hi = torch.cuda.Stream.priority_range()
        level = {"high": hi, "normal": 0, "low": lo}
        self.main = _stream("ticks", level[tick_priority])
        # admitted jobs' host rows go up on their own stream, beside the ticks and the MSMs
        self.copy_stream = _stream("copies", 0)
        # MSM streams pull the pending MSM work whenever their last batch is done; two let
        # one batch's latency-bound tail (bucket reduction, final combination) overlap the
        # next batch's accumulation
        self.msm_streams = [_stream(f"msm{k}", level[msm_priority]) for k in range(max(1, msm_streams))]
        self.msm_last: list[Any] = [None] * len(self.msm_streams)
        self.pending_msm: list[tuple[list, list[int], Any]] = []
        self.msm_batches = 0
        self.max_batch_points = max_batch_points
        self.jobs: dict[int, ProofJob] = {}
        self.records: dict[int, JobRecord] = {}
        self.pending: dict[int, ProofRequest] = {}
        self.tick_events: deque[Any] = deque()
        self.prev_tick_event: Any = None
        self.msm_done: list[tuple[Any, list[int]]] = []  # (event, job ids), in launch order
        self.outstanding: dict[int, int] = {}  # MSM batches of a job not yet complete
        self.ticks = 0
        self.launches = 0

    # ---- footprint ----------------------------------------------------------

    def footprint(self, m: int) -> int:
        """Device bytes one job of size m holds while in flight (computed once per size)."""
        cache = self.__dict__.setdefault("_footprints", {})
        if m not in cache:
            cache[m] = self._footprint(m)
        return cache[m]

    def _footprint(self, m: int) -> int:
        lib = _native.lib()
        buffers = (4 + 3 + 3 + 3 + 1 + 1) * m * 32 + 32 * 5
        ntt_ws = 3 * int(lib.zkb_ntt_workspace_bytes(m))
        jobs = (_native.ZkbMsmJob * 4)()
        for k, n in enumerate((m, m, m - 2, m - 1)):
            jobs[k].points, jobs[k].scalars, jobs[k].n, jobs[k].result = 256, 256, n, 256
            jobs[k].window_size = self.table.window_size if self.table is not None else 0
        msm_ws = int(lib.zkb_msm_fixed_batch_workspace_bytes(jobs, 4) if self.table is not None
                     else lib.zkb_msm_batch_workspace_bytes(jobs, 4))
        return buffers + ntt_ws + msm_ws

    # ---- the loop -----------------------------------------------------------

    def run(self, requests: Sequence[ProofRequest], arrivals_s: Sequence[float],
            clock: Callable[[], float] = time.perf_counter) -> list[JobRecord]:
        """Serve requests[k] arriving arrivals_s[k] seconds after the start (ascending);
        returns one record per job with its arrival, admission and completion times."""
        torch = self.torch
        if len(requests) != len(arrivals_s):
            raise ValueError("one arrival time per request")
        for k, (req, t) in enumerate(zip(requests, arrivals_s, strict=True)):
            self.sched.submit(k, self.footprint(req.m), float(t))
            self.pending[k] = req
            self.records[k] = JobRecord(k, req.m, float(t))
        torch.cuda.synchronize()
        self.start_event = torch.cuda.Event(enable_timing=True)
        self.start_event.record(self.main)
        with torch.cuda.stream(self.main):  # job buffers, uploads and ticks on the tick stream
            t0 = clock()
            while not self.sched.idle():
                now = clock() - t0
                admitted = self.sched.admit(now)
                for job_id in admitted:
                    self.jobs[job_id] = self._new_job(self.pending.pop(job_id), job_id)
                    self.records[job_id].admitted_s = now
                    self.outstanding[job_id] = 0
                tick = self.sched.next_tick(admitted)
                if not tick.empty():
                    self._launch(tick)
                self._dispatch_msm()
                self._collect(block=False)
                if tick.empty():
                    head_waits = bool(self.sched.queue) and self.sched.queue[0][2] > clock() - t0
                    if self.msm_done and not head_waits:
                        # nothing to launch until a job finishes (or frees budget)
                        self._collect(block=True)
                    elif head_waits:
                        wait = self.sched.queue[0][2] - (clock() - t0)
                        time.sleep(max(0.0, min(wait, 0.0005 if self.msm_done else 0.002)))
                while len(self.tick_events) > self.max_ticks_ahead:
                    self.tick_events.popleft().synchronize()
                    self._collect(block=False)
        torch.cuda.synchronize()
        return [self.records[k] for k in range(len(requests))]

    def _new_job(self, request: ProofRequest, job_id: int) -> ProofJob:
        """A job's buffers, from the copy stream's share of the allocator: its rows are written
        on that stream first, so the memory handed to it is never memory that work queued on
        another stream may still use (a block freed on the tick stream while a queued
        transform still reads it would be, if the job were allocated there). The streams that
        use the buffers later are recorded, so the block is reused only after their work."""
        torch = self.torch
        with torch.cuda.stream(self.copy_stream):
            job = ProofJob(request, self.bases, job_id)
        job._mem.record_stream(self.main)
        for stream in self.msm_streams:
            job._mem.record_stream(stream)
        return job

    def _collect(self, block: bool) -> None:
        """Retire jobs whose MSM batches all finished; completion time from the device clock."""
        if block and self.msm_done:
            self.msm_done[0][0].synchronize()
        keep = []
        for ev, ids in self.msm_done:
            if not ev.query():
                keep.append((ev, ids))
                continue
            done_s = self.start_event.elapsed_time(ev) * 1e-3
            for job_id in ids:
                rec = self.records[job_id]
                rec.finished_s = max(rec.finished_s, done_s)
                self.outstanding[job_id] -= 1
        self.msm_done = keep
        for job_id in [j for j, n in self.outstanding.items() if n == 0 and self.sched.stage.get(j) == STAGE_DONE]:
            del self.outstanding[job_id]
            self.sched.finish(job_id)
            self.jobs.pop(job_id)

    def _queue_msm(self, entries: list[tuple[int, int, int, int]], ids: list[int], after: Any) -> None:
        """MSM work becomes pending; an idle MSM stream takes all pending work at once."""
        self.pending_msm.append((entries, list(ids), after))
        for job_id in ids:
            self.outstanding[job_id] += 1

    def _dispatch_msm(self) -> None:
        """Launch pending MSMs as one batch on each MSM stream whose last batch has
        finished: batches grow with the load (up to max_batch_points), so their
        latency-bound tails are shared."""
        torch = self.torch
        lib = _native.lib()
        for k, stream in enumerate(self.msm_streams):
            if not self.pending_msm:
                return
            last = self.msm_last[k]
            if last is not None and not last.query():
                continue
            # first come, first served, up to max_batch_points points (at least one group)
            take, points = 0, 0
            while take < len(self.pending_msm):
                n = sum(e[2] for e in self.pending_msm[take][0])
                if take and points + n > self.max_batch_points:
                    break
                points += n
                take += 1
            work, self.pending_msm = self.pending_msm[:take], self.pending_msm[take:]
            entries = [e for w in work for e in w[0]]
            ids = [j for w in work for j in w[1]]
            if self.table is not None:
                jobs = msm_table_jobs(self.table, entries)
                size_fn, run_fn, name = lib.zkb_msm_fixed_batch_workspace_bytes, lib.zkb_msm_fixed_batch, \
                    "zkb_msm_fixed_batch"
            else:
                jobs = (_native.ZkbMsmJob * len(entries))()
                for j, (pts, sc, n, res) in enumerate(entries):
                    jobs[j].points, jobs[j].scalars, jobs[j].n, jobs[j].result = pts, sc, n, res
                size_fn, run_fn, name = lib.zkb_msm_batch_workspace_bytes, lib.zkb_msm_batch, "zkb_msm_batch"
            for w in work:
                stream.wait_event(w[2])  # the witness / h these MSMs read is written
            before = int(lib.zkb_launch_count())
            with torch.cuda.stream(stream):
                ws_bytes = int(size_fn(jobs, len(entries)))
                ws = _native.workspace(ws_bytes)
                _native.check(run_fn(jobs, len(entries), _native.ptr(ws), ws_bytes, _native.stream_ptr()), name)
                done = torch.cuda.Event(enable_timing=True)
                done.record(stream)
            self.launches += int(lib.zkb_launch_count()) - before
            self.msm_last[k] = done
            self.msm_done.append((done, ids))
            self.msm_batches += 1

    def _launch(self, tick: Tick) -> None:
        torch = self.torch
        lib = _native.lib()
        before = int(lib.zkb_launch_count())
        s = _native.stream_ptr()
        f = ctypes.byref(_native_fr())
        # The admitted jobs' rows go up in groups (as many jobs as one transform launch
        # holds), each with its own event: the copies land while this tick's transforms of
        # resident jobs and the MSM batches run, and a group's own work starts as soon as
        # its rows are on the device, while the next group's copies are still running.
        groups = []
        per = max(1, MAX_NTT_PER_LAUNCH // 3)
        if tick.admitted:
            with torch.cuda.stream(self.copy_stream):
                for lo in range(0, len(tick.admitted), per):
                    ids = tick.admitted[lo : lo + per]
                    for job_id in ids:
                        self.jobs[job_id].copy_rows()
                    event = torch.cuda.Event()
                    event.record(self.copy_stream)
                    groups.append((ids, event))
        for job_id in tick.quotient:
            _native.check(lib.zkb_quotient_pointwise(*self.jobs[job_id].quotient_args(), s),
                          "zkb_quotient_pointwise")
        resident = []
        for stage, ids in ((STAGE_COSET, tick.coset), (STAGE_QUOTIENT, tick.quotient)):
            for job_id in ids:
                resident.extend(self.jobs[job_id].ntt_entries(stage))
        self._ntt_batches(resident, f, s)
        for job_id in tick.quotient:
            self.jobs[job_id].h_to_plain()
        for ids, event in groups:  # the admitted jobs are the tick's INTT stage
            self.main.wait_event(event)
            for job_id in ids:
                self.jobs[job_id].to_montgomery()
            self._ntt_batches([e for j in ids for e in self.jobs[j].ntt_entries(STAGE_INTT)], f, s)
        prev_event = self.prev_tick_event
        tick_event = torch.cuda.Event()
        tick_event.record(self.main)
        self.tick_events.append(tick_event)
        self.prev_tick_event = tick_event
        for ids, event in groups:
            # A, B and L need only the witness: they start once it is copied, beside the quotient
            self._queue_msm([e for j in ids for e in self.jobs[j].msm_entries()[:3]], ids, event)
        if tick.msm:
            # H needs h, written by the previous tick
            self._queue_msm([self.jobs[j].msm_entries()[3] for j in tick.msm], tick.msm, prev_event)
        self.ticks += 1
        self.launches += int(lib.zkb_launch_count()) - before

    def _ntt_batches(self, entries: list, f: Any, s: int) -> None:
        """Transforms (in, out, n, invert, coset) as zkb_ntt_batch launches of up to 64."""
        lib = _native.lib()
        for lo in range(0, len(entries), MAX_NTT_PER_LAUNCH):
            chunk = entries[lo : lo + MAX_NTT_PER_LAUNCH]
            jobs = (_native.ZkbNttJob * len(chunk))()
            for j, (src, dst, n, inv, coset) in enumerate(chunk):
                jobs[j].input, jobs[j].out, jobs[j].n, jobs[j].invert = src, dst, n, int(inv)
                jobs[j].has_coset = int(coset is not None)
                if coset is not None:
                    jobs[j].coset[0] = COSET
            ws_bytes = int(lib.zkb_ntt_batch_workspace_bytes(jobs, len(chunk)))
            ws = _native.workspace(ws_bytes)
            _native.check(lib.zkb_ntt_batch(f, jobs, len(chunk), _native.ptr(ws), ws_bytes, None, s),
                          "zkb_ntt_batch")


_STREAMS: dict[tuple[int, str, int], Any] = {}


def _stream(role: str, priority: int) -> Any:
    """The process's one stream for a role and priority on the current device. Servers reuse
    them: torch's caching allocator hands a freed block out again only on the stream it was
    allocated on, so a server with new streams could use none of the memory its predecessors
    cached, and each run grew the reserved memory (by ~29 GB for 200 queued jobs) until an
    allocation failed and the allocator released its cache behind a full device
    synchronisation."""
    torch = _native.torch_module()
    key = (torch.cuda.current_device(), role, priority)
    if key not in _STREAMS:
        _STREAMS[key] = torch.cuda.Stream(priority=priority)
    return _STREAMS[key]


def _native_fr() -> Any:
    from zkgpu.field256_gpu import BN254_FR

    return BN254_FR._field()


def summarize(records: Sequence[JobRecord], wall_s: float | None = None) -> dict[str, float]:
    """Throughput and latency percentiles of a run."""
    lat = [r.latency_ms for r in records]
    span = wall_s if wall_s is not None else max(r.finished_s for r in records) - min(r.arrival_s for r in records)
    return {
        "jobs": len(records),
        "jobs_per_s": len(records) / span if span > 0 else float("nan"),
        "p50_ms": percentile(lat, 50),
        "p90_ms": percentile(lat, 90),
        "p99_ms": percentile(lat, 99),
        "max_ms": max(lat) if lat else float("nan"),
    }
