"""
zkgpu.sharded — one MSM or one NTT split over several GPUs (one process per
GPU, torch.distributed over NCCL for the exchanges).

The reference runs on one GPU. Its two hot operations shard as follows:

- MSM (msm_sharded): every rank holds a slice of the points and their
  scalars and computes its partial sum with the one-GPU pipeline; the G
  partial sums (72 bytes each) are all-gathered and added. The only exchange
  is that gather.
- NTT (ntt_sharded): n = G m rows, rank r holding x[r m .. r m + m) (block
  layout). Two all-to-all exchanges of (G - 1) / G of the data bracket one
  cross-rank step (zkb_ntt_cross_step: the G-point transforms across ranks
  and the twiddles) and one ordinary m-point NTT (zkb_ntt) per rank. The
  result comes out in cyclic layout, rank t holding y[t], y[t + G], ...;
  cyclic_to_block moves it to block layout with one more exchange. Inverse
  and coset transforms are supported; the results equal BN254_FR.ntt's.

Each rank's side of an algorithm is a generator that yields its exchanges
("all_to_all", tensor) or ("all_gather", tensor) and receives the result. A
driver performs them: run_distributed with torch.distributed (NCCL between
GPUs, or gloo for CPU tests), run_emulated for G ranks inside one process
(each yield handled for all ranks at once), which is how the split algorithms
are checked on a single GPU. The per-rank arithmetic goes through an `ops`
object (GpuOps by default), so the exchange logic can also be tested on the
CPU with other arithmetic.
"""

from __future__ import annotations

import ctypes
from collections.abc import Generator, Sequence
from typing import Any

import numpy as np

from zkgpu import _native
from zkgpu.curve import R, Point
from zkgpu.field256_gpu import BN254_FR, LIMBS

COSET_DEFAULT = 5
_MONT_R = (1 << 256) % R

Exchange = Generator[tuple[str, Any], Any, Any]


def _mont_rows(values: Sequence[int]) -> list[list[int]]:
    return [_native.limbs(v * _MONT_R % R) for v in values]


class GpuOps:
    """Per-rank arithmetic on this process's GPU through libzkb200.so."""

    def __init__(self) -> None:
        self.torch = _native.require_cuda()

    def cross_step(self, recv: Any, n: int, parts: int, part: int, invert: bool, coset: int | None) -> Any:
        torch = self.torch
        lib = _native.lib()
        out = torch.empty_like(recv)
        post = None
        if invert:  # G^-1 g^-k1 for output block k1, in Montgomery form
            g_inv = pow(coset, -1, R) if coset is not None else 1
            g_part_inv = pow(parts, -1, R)
            rows = _mont_rows([g_part_inv * pow(g_inv, k, R) % R for k in range(parts)])
            post = torch.from_numpy(np.array(rows, dtype=np.uint64).view(np.int64)).to(recv.device)
        g = _native.u64_array(_native.limbs(coset % R)) if (coset is not None and not invert) else None
        _native.check(lib.zkb_ntt_cross_step(ctypes.byref(BN254_FR._field()), _native.ptr(recv), _native.ptr(out),
                                             n, parts, part, int(invert), g,
                                             _native.ptr(post) if post is not None else None,
                                             _native.stream_ptr()), "zkb_ntt_cross_step")
        return out

    def ntt(self, rows: Any, invert: bool, coset: int | None) -> Any:
        return BN254_FR.ntt(rows, invert=invert, coset=coset)

    def msm(self, points: Any, scalars: Any, window_size: int | None) -> Any:
        torch = self.torch
        lib = _native.lib()
        n = int(points.shape[0])
        out = torch.zeros(16, dtype=torch.int64, device=points.device)
        if n == 0:
            out[8] = 1
            return out
        w = 0 if window_size is None else int(window_size)
        ws_bytes = lib.zkb_msm_workspace_bytes(n, w)
        ws = _native.workspace(ws_bytes)
        _native.check(lib.zkb_msm(_native.ptr(points), _native.ptr(scalars), n, w, _native.ptr(out),
                                  _native.ptr(ws), ws_bytes, _native.stream_ptr()), "zkb_msm")
        return out

    def combine(self, partials: Any) -> Point:
        from zkgpu.batch import results_to_points

        total = Point.identity()
        for p in results_to_points(partials):
            total = total + p
        return total


# ------------------------------------------------------------------
# Per-rank algorithms (generators)
# ------------------------------------------------------------------


def _check_split(n: int, parts: int) -> None:
    if parts < 1 or parts & (parts - 1) or parts > 16:
        raise ValueError(f"parts must be a power of 2 up to 16, got {parts}")
    if n & (n - 1) or n < parts * parts or n > 1 << 28:
        raise ValueError(f"NTT length must be a power of 2 with parts^2 <= n <= 2^28, got {n} for {parts} parts")


def ntt_rank(x_local: Any, parts: int, rank: int, *, invert: bool = False, coset: int | None = None,
             ops: Any = None) -> Exchange:
    """Rank `rank`'s side of an n = parts * len(x_local) point NTT: block layout in,
    cyclic layout out (rank t ends with y[t + k parts] for k < n / parts)."""
    m = int(x_local.shape[0])
    n = m * parts
    _check_split(n, parts)
    if coset is not None and coset % R == 0:
        raise ValueError(f"coset offset {coset} must be non-zero")
    ops = ops or GpuOps()
    if parts == 1:
        return ops.ntt(x_local, invert, coset)
    c = m // parts
    recv = yield ("all_to_all", x_local.reshape(parts, c, LIMBS))
    out = ops.cross_step(recv.reshape(parts * c, LIMBS), n, parts, rank, invert, coset)
    recv2 = yield ("all_to_all", out.reshape(parts, c, LIMBS))
    local_coset = pow(coset, parts, R) if (coset is not None and invert) else None
    return ops.ntt(recv2.reshape(m, LIMBS), invert, local_coset)


def cyclic_to_block_rank(y_local: Any, parts: int, rank: int) -> Exchange:
    """Rank `rank`'s side of the move from cyclic layout (y[rank + k parts]) to block layout
    (y[rank m .. rank m + m)). `rank` is implied by the exchange; it is kept for symmetry."""
    del rank
    if parts == 1:
        return y_local
    m = int(y_local.shape[0])
    c = m // parts
    # to rank t go the entries k in [t c, (t + 1) c): y[r + k parts] lands in t's block
    recv = yield ("all_to_all", y_local.reshape(parts, c, LIMBS))
    # recv[r][i] = y[r + (t c + i) parts]: interleave the sources
    return recv.permute(1, 0, 2).reshape(m, LIMBS).contiguous()


def msm_rank(points_local: Any, scalars_local: Any, *, window_size: int | None = None,
             ops: Any = None) -> Exchange:
    """Rank's side of a point-sharded MSM: its partial sum, all-gathered and added."""
    ops = ops or GpuOps()
    partial = ops.msm(points_local, scalars_local, window_size)
    everyone = yield ("all_gather", partial)
    return ops.combine(everyone)


# ------------------------------------------------------------------
# Drivers
# ------------------------------------------------------------------


def run_distributed(gen: Exchange, group: Any = None) -> Any:
    """Drive one rank's generator with torch.distributed collectives (NCCL or gloo)."""
    import torch
    import torch.distributed as dist

    try:
        op, t = next(gen)
        while True:
            t = t.contiguous()
            if op == "all_to_all":
                recv = torch.empty_like(t)
                dist.all_to_all_single(recv, t, group=group)
            elif op == "all_gather":
                world = dist.get_world_size(group)
                flat = torch.empty(world * t.numel(), dtype=t.dtype, device=t.device)
                dist.all_gather_into_tensor(flat, t.reshape(-1), group=group)
                recv = flat.view(world, *t.shape)
            else:
                raise ValueError(f"unknown exchange {op}")
            op, t = gen.send(recv)
    except StopIteration as done:
        return done.value


def run_emulated(gens: Sequence[Exchange]) -> list[Any]:
    """Drive G ranks' generators in one process: all_to_all gives rank r the blocks
    [s][r] of every rank s, all_gather stacks every rank's tensor."""
    import torch

    results: list[Any] = [None] * len(gens)
    live = list(range(len(gens)))
    msgs: dict[int, tuple[str, Any]] = {}
    for r in live:
        try:
            msgs[r] = next(gens[r])
        except StopIteration as done:
            results[r] = done.value
    live = [r for r in live if r in msgs]
    while live:
        ops = {msgs[r][0] for r in live}
        if len(ops) != 1 or len(live) != len(gens):
            raise RuntimeError("ranks disagree on the exchange sequence")
        op = ops.pop()
        sends = [msgs[r][1] for r in live]
        if op == "all_to_all":
            replies = [torch.stack([sends[s][r] for s in range(len(sends))]) for r in range(len(sends))]
        elif op == "all_gather":
            stacked = torch.stack(sends)
            replies = [stacked.clone() for _ in sends]
        else:
            raise ValueError(f"unknown exchange {op}")
        nxt = {}
        for r, reply in zip(live, replies, strict=True):
            try:
                nxt[r] = gens[r].send(reply)
            except StopIteration as done:
                results[r] = done.value
        live = [r for r in live if r in nxt]
        msgs = nxt
    return results


# ------------------------------------------------------------------
# Whole-job helpers over torch.distributed
# ------------------------------------------------------------------


def ntt_sharded(x_local: Any, *, invert: bool = False, coset: int | None = None, group: Any = None,
                block_output: bool = False) -> Any:
    """This rank's part of the NTT of the rows every rank's x_local make up in rank order.
    Cyclic output layout unless block_output (one more exchange)."""
    import torch.distributed as dist

    parts, rank = dist.get_world_size(group), dist.get_rank(group)
    y = run_distributed(ntt_rank(x_local, parts, rank, invert=invert, coset=coset), group)
    return run_distributed(cyclic_to_block_rank(y, parts, rank), group) if block_output else y


def msm_sharded(points_local: Any, scalars_local: Any, *, window_size: int | None = None,
                group: Any = None) -> Point:
    """sum s_i P_i over the points and scalars of every rank (each rank its slice)."""
    return run_distributed(msm_rank(points_local, scalars_local, window_size=window_size), group)


def shard_bounds(n: int, parts: int, rank: int) -> tuple[int, int]:
    """[lo, hi) of rank's contiguous share of n items (the first n % parts ranks get one more)."""
    base, extra = divmod(n, parts)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


__all__ = [
    "GpuOps", "cyclic_to_block_rank", "msm_rank", "msm_sharded", "ntt_rank", "ntt_sharded", "run_distributed",
    "run_emulated", "shard_bounds",
]
