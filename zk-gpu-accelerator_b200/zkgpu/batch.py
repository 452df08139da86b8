"""
zkgpu.batch — many NTTs and MSMs per launch, and CUDA-graph replay of
repeated shapes.

The reference runs one transform or one MSM per call (Field256.ntt,
msm_pippenger_gpu). A prover and a proving service run many of uneven sizes;
this module batches them:

- ntt_batch: up to 64 BN254 Fr transforms (forward, inverse, coset) in one
  persistent kernel launch fed by a device tile counter (zkb_ntt_batch);
- msm_batch: any number of G1 MSMs (zkb_msm_batch): jobs of one window size
  share one sort / bucket / reduction / finalize pipeline, groups of
  different window sizes run concurrently on side streams;
- BatchPlan: a fixed set of NTT and MSM jobs over bound device buffers, with
  its workspace and outputs allocated once, that can be captured into a CUDA
  graph and replayed (new inputs are copied into the bound buffers first).

Every result is bit-identical to the one-at-a-time call with the same
arguments (Field256.ntt, msm_pippenger_rows).
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence
from typing import Any

import numpy as np

from zkgpu import _native, _rows
from zkgpu.curve import R as _GROUP_ORDER, Point
from zkgpu.field256_gpu import BN254_FR, LIMBS

MAX_NTT_BATCH = 64
_RESULT_WORDS = 16  # 9 result words padded to 128-byte rows


def _is_pow2(n: int) -> bool:
    return n >= 0 and (n & (n - 1)) == 0


def _ntt_jobs(inputs: Sequence[Any], outputs: Sequence[Any], invert: Sequence[bool],
              coset: Sequence[int | None]) -> Any:
    arr = (_native.ZkbNttJob * max(len(inputs), 1))()
    for j, (x, y, inv, g) in enumerate(zip(inputs, outputs, invert, coset, strict=True)):
        arr[j].input = _native.ptr(x)
        arr[j].out = _native.ptr(y)
        arr[j].n = int(x.shape[0])
        arr[j].invert = int(bool(inv))
        arr[j].has_coset = int(g is not None)
        if g is not None:
            for k, v in enumerate(_native.limbs(g % _GROUP_ORDER)):
                arr[j].coset[k] = v
    return arr


def _msm_jobs(points: Sequence[Any], scalars: Sequence[Any], results: Any,
              window_sizes: Sequence[int | None], counts: Sequence[int] | None = None) -> Any:
    arr = (_native.ZkbMsmJob * max(len(points), 1))()
    for j, (p, s, w) in enumerate(zip(points, scalars, window_sizes, strict=True)):
        arr[j].points = _native.ptr(p)
        arr[j].scalars = _native.ptr(s)
        arr[j].n = int(p.shape[0]) if counts is None else int(counts[j])
        arr[j].result = _native.ptr(results) + 8 * _RESULT_WORDS * j
        arr[j].window_size = 0 if w is None else int(w)
    return arr


def _check_ntt_inputs(xs: Sequence[Any], invert: Any, coset: Any) -> tuple[list[bool], list[int | None]]:
    if len(xs) > MAX_NTT_BATCH:
        raise ValueError(f"an NTT batch holds at most {MAX_NTT_BATCH} transforms, got {len(xs)}")
    inv = list(invert) if isinstance(invert, (list, tuple)) else [bool(invert)] * len(xs)
    cos = list(coset) if isinstance(coset, (list, tuple)) else [coset] * len(xs)
    if len(inv) != len(xs) or len(cos) != len(xs):
        raise ValueError(f"Length mismatch: {len(xs)} inputs, {len(inv)} invert flags, {len(cos)} cosets.")
    for x in xs:
        if not _rows.shape_ok(x, (LIMBS,)):
            raise TypeError(f"NTT inputs must be (n, 4) uint64 arrays, got {_rows._describe(x)}")
        n = int(x.shape[0])
        if not _is_pow2(n):
            raise ValueError(f"NTT length must be a power of 2, got {n}")
        if n > 1 << 28:
            raise ValueError(f"NTT length {n} not supported (at most 2^28 for BN254 Fr)")
    for g in cos:
        if g is not None and g % _GROUP_ORDER == 0:
            raise ValueError(f"coset offset {g} must be non-zero")
    return inv, cos


def ntt_batch(xs: Sequence[Any], *, invert: bool | Sequence[bool] = False,
              coset: int | None | Sequence[int | None] = None) -> list[Any]:
    """
    BN254 Fr NTTs of Montgomery rows xs[j] (each (n_j, 4), n_j a power of two),
    in one persistent launch; returns new output rows per job. `invert` and
    `coset` apply to every job, or give one value per job. Same results as
    BN254_FR.ntt(xs[j], invert=..., coset=...).
    """
    torch = _native.require_cuda()
    inv, cos = _check_ntt_inputs(xs, invert, coset)
    ins = [_rows.to_device(x) for x in xs]
    outs = [_rows.empty((int(x.shape[0]), LIMBS)) for x in ins]
    if not ins:
        return []
    jobs = _ntt_jobs(ins, outs, inv, cos)
    lib = _native.lib()
    ws_bytes = lib.zkb_ntt_batch_workspace_bytes(jobs, len(ins))
    if ws_bytes == 0:
        raise RuntimeError(_native.last_error() or "zkb_ntt_batch_workspace_bytes failed")
    ws = _native.workspace(ws_bytes)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _native.check(lib.zkb_ntt_batch(ctypes.byref(BN254_FR._field()), jobs, len(ins), _native.ptr(ws), ws_bytes,
                                    _native.ptr(status), _native.stream_ptr()), "zkb_ntt_batch")
    _native.check(int(status.item()), "zkb_ntt_batch (device status)")
    return outs


def msm_batch(points: Sequence[Any], scalars: Sequence[Any], *,
              window_sizes: Sequence[int | None] | None = None) -> list[Point]:
    """
    sum_i s_i P_i for every job j: points[j] (n_j, 2, 4) Montgomery affine rows
    (e.g. a prefix of one resident base set), scalars[j] (n_j, 4) limb rows.
    Same results as msm_pippenger_rows(points[j], scalars[j], check_points=False).
    """
    torch = _native.require_cuda()
    if len(points) != len(scalars):
        raise ValueError(f"Length mismatch: {len(points)} point sets, {len(scalars)} scalar sets.")
    ws_list = list(window_sizes) if window_sizes is not None else [None] * len(points)
    if len(ws_list) != len(points):
        raise ValueError(f"Length mismatch: {len(points)} jobs, {len(ws_list)} window sizes.")
    pts = [_rows.to_device(p) for p in points]
    scs = [_rows.to_device(s) for s in scalars]
    for p, s in zip(pts, scs, strict=True):
        if not _rows.shape_ok(p, (2, LIMBS)):
            raise TypeError(f"points must be an (n, 2, 4) uint64 array of affine points, got {_rows._describe(p)}")
        if not _rows.shape_ok(s, (LIMBS,)):
            raise TypeError(f"scalars must be an (n, 4) uint64 array of limbs, got {_rows._describe(s)}")
        if int(p.shape[0]) != int(s.shape[0]):
            raise ValueError(f"Length mismatch: {int(p.shape[0])} points, {int(s.shape[0])} scalars.")
    if not pts:
        return []
    results = torch.empty((len(pts), _RESULT_WORDS), dtype=torch.int64, device="cuda")
    jobs = _msm_jobs(pts, scs, results, ws_list)
    lib = _native.lib()
    ws_bytes = lib.zkb_msm_batch_workspace_bytes(jobs, len(pts))
    err = _native.last_error()
    if err:
        raise ValueError(err)
    ws = _native.workspace(ws_bytes)
    _native.check(lib.zkb_msm_batch(jobs, len(pts), _native.ptr(ws), ws_bytes, _native.stream_ptr()),
                  "zkb_msm_batch")
    return results_to_points(results)


def msm_fixed_batch(table: Any, scalars: Sequence[Any]) -> list[Point]:
    """
    sum_i s_i P_i for every job j over the first len(scalars[j]) points of a
    FixedBaseTable (zkb_msm_fixed_batch): one pipeline for all jobs. Same
    results as msm_batch over the table's points.
    """
    torch = _native.require_cuda()
    scs = [_rows.to_device(s) for s in scalars]
    for s in scs:
        if not _rows.shape_ok(s, (LIMBS,)):
            raise TypeError(f"scalars must be an (n, 4) uint64 array of limbs, got {_rows._describe(s)}")
        if int(s.shape[0]) > table.n:
            raise ValueError(f"Length mismatch: {int(s.shape[0])} scalars for a table of {table.n} points.")
    if not scs:
        return []
    results = torch.empty((len(scs), _RESULT_WORDS), dtype=torch.int64, device="cuda")
    jobs = (_native.ZkbMsmJob * len(scs))()
    for j, s in enumerate(scs):
        jobs[j].points = _native.ptr(table.table)
        jobs[j].scalars = _native.ptr(s)
        jobs[j].n = int(s.shape[0])
        jobs[j].result = _native.ptr(results) + 8 * _RESULT_WORDS * j
        jobs[j].window_size = table.window_size
    lib = _native.lib()
    ws_bytes = lib.zkb_msm_fixed_batch_workspace_bytes(jobs, len(scs))
    err = _native.last_error()
    if err:
        raise ValueError(err)
    ws = _native.workspace(ws_bytes)
    _native.check(lib.zkb_msm_fixed_batch(jobs, len(scs), _native.ptr(ws), ws_bytes, _native.stream_ptr()),
                  "zkb_msm_fixed_batch")
    return results_to_points(results)


def results_to_points(results: Any) -> list[Point]:
    """Points of an (m, 16) int64 result block (zkb_msm's 9 words per row)."""
    from zkgpu.msm_gpu import _result_point

    host = results.to("cpu").numpy().view(np.uint64)
    return [_result_point(host[j, :9]) for j in range(host.shape[0])]


class BatchPlan:
    """
    A fixed set of NTT jobs and MSM jobs over bound device buffers, launched
    together: NTTs through one zkb_ntt_batch launch, MSMs through one
    zkb_msm_batch call, both on the current stream. Outputs and workspaces
    are allocated once, so run() allocates nothing and can be captured into a
    CUDA graph (capture()) and replayed (replay()) for repeated shapes; to
    process new data, copy it into the bound input tensors first.

    ntt_jobs : [(rows, invert, coset)] with rows (n, 4) Montgomery, device
    msm_jobs : [(points, scalars, window_size)] device tensors
    table    : optional FixedBaseTable of a resident base set whose prefixes every
               MSM job's points are: the MSMs then run over the table
               (zkb_msm_fixed_batch, one bucket set per job, no final doublings;
               the table's window replaces the jobs'), with the same results
    concurrent : run the MSM batch on a high-priority stream and the transforms,
                 one pass launch at a time (zkb_ntt per job), on a low-priority
                 stream beside it. The block scheduler then hands SMs to NTT
                 blocks whenever the MSM kernels have none waiting: during the
                 memory-bound sort, the tail of every wave and the
                 latency-bound bucket reduction and final combination, so
                 those overlap the transforms. run() still returns with all
                 the work ordered on the current stream.
    """

    def __init__(self, ntt_jobs: Sequence[tuple[Any, bool, int | None]] = (),
                 msm_jobs: Sequence[tuple[Any, Any, int | None]] = (), concurrent: bool = False,
                 table: Any = None) -> None:
        torch = _native.require_cuda()
        self._torch = torch
        self._concurrent = concurrent
        if concurrent:
            lo, hi = torch.cuda.Stream.priority_range()
            self._hi = torch.cuda.Stream(priority=hi)
            self._lo = torch.cuda.Stream(priority=lo)
            self._ntt_single_ws = [_native.workspace(_native.lib().zkb_ntt_workspace_bytes(int(j[0].shape[0])))
                                   for j in ntt_jobs]
        lib = _native.lib()
        xs = [j[0] for j in ntt_jobs]
        inv, cos = _check_ntt_inputs(xs, [j[1] for j in ntt_jobs], [j[2] for j in ntt_jobs])
        self.ntt_inputs = list(xs)
        self.ntt_outputs = [_rows.empty((int(x.shape[0]), LIMBS)) for x in xs]
        self._ntt = _ntt_jobs(self.ntt_inputs, self.ntt_outputs, inv, cos) if xs else None
        self._ntt_count = len(xs)
        self._ntt_ws_bytes = lib.zkb_ntt_batch_workspace_bytes(self._ntt, len(xs)) if xs else 0
        if xs and self._ntt_ws_bytes == 0:
            raise RuntimeError(_native.last_error() or "zkb_ntt_batch_workspace_bytes failed")
        self._ntt_ws = _native.workspace(self._ntt_ws_bytes)
        self.status = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.msm_points = [j[0] for j in msm_jobs]
        self.msm_scalars = [j[1] for j in msm_jobs]
        self.msm_results = torch.zeros((max(len(msm_jobs), 1), _RESULT_WORDS), dtype=torch.int64,
                                       device="cuda")
        self._msm_count = len(msm_jobs)
        self._table = table
        if table is not None:
            for p in self.msm_points:
                if int(p.shape[0]) > table.n:
                    raise ValueError(f"an MSM of {int(p.shape[0])} points over a table of {table.n}")
            self._msm = (_msm_jobs([table.table] * len(msm_jobs), self.msm_scalars, self.msm_results,
                                   [table.window_size] * len(msm_jobs), [int(p.shape[0]) for p in self.msm_points])
                         if msm_jobs else None)
            self._msm_ws_bytes = lib.zkb_msm_fixed_batch_workspace_bytes(self._msm, len(msm_jobs)) if msm_jobs else 0
        else:
            self._msm = (_msm_jobs(self.msm_points, self.msm_scalars, self.msm_results,
                                   [j[2] for j in msm_jobs]) if msm_jobs else None)
            self._msm_ws_bytes = lib.zkb_msm_batch_workspace_bytes(self._msm, len(msm_jobs)) if msm_jobs else 0
        if msm_jobs and _native.last_error():
            raise ValueError(_native.last_error())
        self._msm_ws = _native.workspace(self._msm_ws_bytes)
        self._graph = None
        self.launches_per_run = 0

    def run(self) -> None:
        """Queue every job on the current stream (asynchronous)."""
        torch = self._torch
        lib = _native.lib()
        main = torch.cuda.current_stream()
        before = int(lib.zkb_launch_count())
        split = self._concurrent and self._ntt_count and self._msm_count
        ntt_stream, msm_stream = (self._lo, self._hi) if split else (main, main)
        if split:
            self._lo.wait_stream(main)
            self._hi.wait_stream(main)
            f = BN254_FR._field()
            for k in range(self._ntt_count):
                j = self._ntt[k]
                g = _native.u64_array(list(j.coset)) if j.has_coset else None
                ws = self._ntt_single_ws[k]
                _native.check(lib.zkb_ntt(ctypes.byref(f), j.input, j.out, j.n, j.invert, None, g,
                                          _native.ptr(ws), ws.numel(), int(ntt_stream.cuda_stream)), "zkb_ntt")
        elif self._ntt_count:
            _native.check(lib.zkb_ntt_batch(ctypes.byref(BN254_FR._field()), self._ntt, self._ntt_count,
                                            _native.ptr(self._ntt_ws), self._ntt_ws_bytes,
                                            _native.ptr(self.status), int(ntt_stream.cuda_stream)),
                          "zkb_ntt_batch")
        if self._msm_count:
            run_fn = lib.zkb_msm_fixed_batch if self._table is not None else lib.zkb_msm_batch
            _native.check(run_fn(self._msm, self._msm_count, _native.ptr(self._msm_ws), self._msm_ws_bytes,
                                 int(msm_stream.cuda_stream)), "zkb_msm_batch")
        if split:
            main.wait_stream(self._lo)
            main.wait_stream(self._hi)
        self.launches_per_run = int(lib.zkb_launch_count()) - before

    def capture(self) -> None:
        """Record run() into a CUDA graph (after one eager run, which builds the NTT tables)."""
        torch = self._torch
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.run()  # warm-up: builds tables, plans and CUB's kernels outside the capture
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.run()
        self._graph = graph

    def replay(self) -> None:
        if self._graph is None:
            raise RuntimeError("BatchPlan.replay() needs capture() first")
        self._graph.replay()

    def check_status(self) -> None:
        """Raise if a bounded wait inside the NTT batch gave up (synchronises)."""
        _native.check(int(self.status.item()), "zkb_ntt_batch (device status)")

    def msm_points_out(self) -> list[Point]:
        return results_to_points(self.msm_results[: self._msm_count])
