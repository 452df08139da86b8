"""
zkgpu.autotune — measured per-size choices for the MSM window and the NTT
pass shape, cached per GPU model and library version.

The reference picks the Pippenger window from an addition-count model
(pippenger_window_size, zkgpu/msm.py:112-121) and has one NTT shape. Here
both are measured: for every log2 size asked for, each candidate is timed
with CUDA events on this GPU (the median of a few runs after a warm-up), and
the fastest goes into the library's per-size tables (zkb_tune_set_sized),
which every later call, batched or not, plans with:

  msm.window                      the default window of an MSM of 2^log points
  ntt.max_log_radix / ntt.cta_log_elems / ntt.threads
                                  the pass split, tile and block of an NTT of 2^log rows

A choice changes only speed: every candidate computes the same rows and
points (the GPU tests check the NTT plans and windows against the
reference). The table is saved as JSON (default ~/.cache/zkgpu/tune.json,
or $ZKGPU_TUNE_CACHE) under a key naming the GPU, its compute capability and
the library's ABI version, and autotune() reuses it when the key matches.
"""

from __future__ import annotations

import json
import os
import statistics
from pathlib import Path
from typing import Any

from zkgpu import _native

CACHE_ENV = "ZKGPU_TUNE_CACHE"
NTT_KEYS = ("ntt.max_log_radix", "ntt.cta_log_elems", "ntt.threads")
MSM_KEY = "msm.window"


def default_cache_path() -> Path:
    return Path(os.environ.get(CACHE_ENV) or Path.home() / ".cache" / "zkgpu" / "tune.json")


def device_key() -> str:
    torch = _native.require_cuda()
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}|sm_{p.major}{p.minor}|{p.multi_processor_count} SMs|abi {_native.lib().zkb_version()}"


def _median_ms(fn, reps: int) -> float:
    torch = _native.torch_module()
    fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
    return statistics.median(times)


# ------------------------------------------------------------------
# MSM window
# ------------------------------------------------------------------


def tune_msm(log_sizes, *, reps: int = 3, spread: int = 2, seed: int = 1) -> dict[int, dict[str, Any]]:
    """Best window per log2 point count (uniform scalars: the costly case), trying the
    library's default window and `spread` on each side."""
    torch = _native.require_cuda()
    from zkgpu import curve_gpu, workloads as wl

    lib = _native.lib()
    logs = sorted(set(int(v) for v in log_sizes))
    if not logs:
        return {}
    n_max = 1 << logs[-1]
    bases = curve_gpu.mul_generator(wl.base_scalars(seed, n_max))
    scalars = torch.from_numpy(wl.uniform_fr(seed + 1, n_max)).cuda()
    out = torch.empty(16, dtype=torch.int64, device="cuda")
    table: dict[int, dict[str, Any]] = {}
    for lg in logs:
        n = 1 << lg
        _native.tune_set_sized(MSM_KEY, lg, 0)  # measure around the model's own choice
        w0 = int(lib.zkb_msm_default_window(n))
        cands = [w for w in range(w0 - spread, w0 + spread + 1) if 1 <= w <= 20]
        times = {}
        for w in cands:
            ws_bytes = int(lib.zkb_msm_workspace_bytes(n, w))
            ws = _native.workspace(ws_bytes)

            def run(w=w, ws=ws, ws_bytes=ws_bytes) -> None:
                _native.check(lib.zkb_msm(bases.data_ptr(), scalars.data_ptr(), n, w, out.data_ptr(),
                                          ws.data_ptr(), ws_bytes, _native.stream_ptr()), "zkb_msm")

            times[w] = _median_ms(run, reps)
            del ws
        best = min(times, key=times.get)
        table[lg] = {"window": best, "ms": round(times[best], 4), "model_window": w0,
                     "candidates_ms": {str(k): round(v, 4) for k, v in times.items()}}
    return table


# ------------------------------------------------------------------
# NTT pass shape
# ------------------------------------------------------------------


def _ntt_candidates(lg: int) -> list[tuple[int, int, int]]:
    cands = []
    for radix in (12, 11, 10, 8):
        if radix < 12 and (lg + radix - 1) // radix == (lg + 11) // 12:
            continue  # the same number of passes as 12-bit ones: same plan
        for cta, threads in ((12, 512), (11, 256), (10, 256), (9, 128)):
            cands.append((radix, cta, threads))
    return cands


def tune_ntt(log_sizes, *, reps: int = 5, seed: int = 2) -> dict[int, dict[str, Any]]:
    """Best (max pass radix, rows per block, threads) per log2 NTT size (forward transforms)."""
    torch = _native.require_cuda()
    from zkgpu import workloads as wl
    from zkgpu.field256_gpu import BN254_FR

    import ctypes

    lib = _native.lib()
    f = BN254_FR._field()
    table: dict[int, dict[str, Any]] = {}
    for lg in sorted(set(int(v) for v in log_sizes)):
        n = 1 << lg
        x = BN254_FR.to_montgomery(wl.uniform_fr(seed + lg, n))
        y = torch.empty_like(x)
        times = {}
        for radix, cta, threads in _ntt_candidates(lg):
            for key, v in zip(NTT_KEYS, (radix, cta, threads), strict=True):
                _native.tune_set_sized(key, lg, v)
            ws_bytes = int(lib.zkb_ntt_workspace_bytes(n))
            ws = _native.workspace(ws_bytes)

            def run(ws=ws, ws_bytes=ws_bytes) -> None:
                _native.check(lib.zkb_ntt(ctypes.byref(f), x.data_ptr(), y.data_ptr(), n, 0, None, None,
                                          ws.data_ptr(), ws_bytes, _native.stream_ptr()), "zkb_ntt")

            times[(radix, cta, threads)] = _median_ms(run, reps)
        for key in NTT_KEYS:
            _native.tune_set_sized(key, lg, 0)
        best = min(times, key=times.get)
        table[lg] = {"max_log_radix": best[0], "cta_log_elems": best[1], "threads": best[2],
                     "ms": round(times[best], 4),
                     "candidates_ms": {"/".join(map(str, k)): round(v, 4) for k, v in times.items()}}
    return table


# ------------------------------------------------------------------
# Tables: apply, save, load
# ------------------------------------------------------------------


def apply(table: dict[str, Any]) -> None:
    """Load a table (as returned by measure / load) into the library."""
    for lg, e in table.get("msm", {}).items():
        _native.tune_set_sized(MSM_KEY, int(lg), int(e["window"]))
    for lg, e in table.get("ntt", {}).items():
        _native.tune_set_sized("ntt.max_log_radix", int(lg), int(e["max_log_radix"]))
        _native.tune_set_sized("ntt.cta_log_elems", int(lg), int(e["cta_log_elems"]))
        _native.tune_set_sized("ntt.threads", int(lg), int(e["threads"]))


def clear() -> None:
    """Remove every per-size entry (back to the built-in rules)."""
    for lg in range(33):
        for key in (MSM_KEY, *NTT_KEYS):
            _native.tune_set_sized(key, lg, 0)


def measure(msm_logs=range(10, 23), ntt_logs=range(10, 25)) -> dict[str, Any]:
    return {"device": device_key(), "msm": tune_msm(msm_logs), "ntt": tune_ntt(ntt_logs)}


def save(table: dict[str, Any], path: str | Path | None = None) -> Path:
    p = Path(path) if path is not None else default_cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    entries = {}
    if p.exists():
        try:
            entries = json.loads(p.read_text())
        except ValueError:
            entries = {}
    entries[table["device"]] = {"msm": {str(k): v for k, v in table["msm"].items()},
                                "ntt": {str(k): v for k, v in table["ntt"].items()}}
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(entries, indent=1, sort_keys=True))
    tmp.replace(p)
    return p


def load(path: str | Path | None = None, key: str | None = None) -> dict[str, Any] | None:
    """The cached table for this device (or `key`), or None."""
    p = Path(path) if path is not None else default_cache_path()
    if not p.exists():
        return None
    try:
        entries = json.loads(p.read_text())
    except ValueError:
        return None
    k = key if key is not None else device_key()
    e = entries.get(k)
    return None if e is None else {"device": k, **e}


def autotune(msm_logs=range(10, 23), ntt_logs=range(10, 25), path: str | Path | None = None,
             force: bool = False) -> dict[str, Any]:
    """Apply the cached table for this device, measuring (and caching) it first when there is
    none, when `force`, or when it lacks a size asked for."""
    table = None if force else load(path)
    if table is not None:
        have_msm = {int(k) for k in table.get("msm", {})}
        have_ntt = {int(k) for k in table.get("ntt", {})}
        if not set(msm_logs) <= have_msm or not set(ntt_logs) <= have_ntt:
            table = None
    if table is None:
        table = measure(msm_logs, ntt_logs)
        save(table, path)
    apply(table)
    return table
