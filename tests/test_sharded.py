"""
The split MSM and NTT (zkgpu.sharded) without a GPU: the exchange logic of
every rank, driven by two gloo processes (torch.distributed, world size 2)
and by the in-process emulation for 2..16 ranks, with the per-rank arithmetic
done by the oracle (the C port's NTT and Pippenger, and a Python-integer
restatement of the cross-rank step). The results must equal the one-piece
transform / MSM of the oracle. The same generators run on the GPU with the
library's arithmetic in tests/test_sharded_gpu.py.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import c_oracle as co
from oracle import pyoracle as po
from zkgpu import sharded
from zkgpu import workloads as wl

R = po.R


def _to_ints(rows: np.ndarray) -> list[int]:
    return wl.rows_to_ints(np.ascontiguousarray(rows, dtype=np.uint64))


def _to_rows(values: list[int]) -> np.ndarray:
    return np.array([[(v >> (64 * j)) & (2**64 - 1) for j in range(4)] for v in values], dtype=np.uint64)


def _t(rows: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(rows, dtype=np.uint64).view(np.int64))


def _np(t: torch.Tensor) -> np.ndarray:
    return t.contiguous().numpy().view(np.uint64)


class OracleOps:
    """Per-rank arithmetic on the CPU: Montgomery rows in and out, as on the GPU."""

    def cross_step(self, recv, n, parts, part, invert, coset):
        m, c = n // parts, n // parts // parts
        w_n = po.get_ntt_root(n, R)
        if invert:
            w_n = pow(w_n, -1, R)
        w_g = pow(w_n, m, R)
        vals = [po.from_mont(v, R) for v in _to_ints(_np(recv))]  # block j1, row i at j1 c + i
        out = [0] * (parts * c)
        for i in range(c):
            j2 = part * c + i
            col = [vals[j1 * c + i] for j1 in range(parts)]
            if coset is not None and not invert:
                col = [v * pow(coset, j1 * m + j2, R) % R for j1, v in enumerate(col)]
            for k1 in range(parts):
                s = sum(v * pow(w_g, j1 * k1, R) for j1, v in enumerate(col)) % R
                s = s * pow(w_n, j2 * k1, R) % R
                if invert:
                    g_inv = pow(coset, -1, R) if coset is not None else 1
                    s = s * pow(parts, -1, R) * pow(g_inv, k1, R) % R
                out[k1 * c + i] = po.to_mont(s, R)
        return _t(_to_rows(out))

    def ntt(self, rows, invert, coset):
        return _t(co.ntt(_np(rows), invert=invert, coset=coset))

    def msm(self, points, scalars, window_size):
        out = np.zeros(16, dtype=np.uint64)
        if points.shape[0] == 0:
            out[8] = 1
        else:
            out[:9] = co.msm(_np(points).reshape(-1, 2, 4), _np(scalars), window_size or 8)
        return _t(out)

    def combine(self, partials):
        total = None
        for row in _np(partials):
            if row[8]:
                continue
            p = tuple(_to_ints(row[:8].reshape(2, 4)))
            total = p if total is None else po.affine_add(total, p)
        return total


def _assemble_cyclic(parts_out: list[torch.Tensor]) -> np.ndarray:
    g = len(parts_out)
    m = parts_out[0].shape[0]
    full = np.empty((g * m, 4), dtype=np.uint64)
    for t, y in enumerate(parts_out):
        full[t::g] = _np(y)
    return full


@pytest.mark.parametrize("parts", [2, 4, 8, 16])
@pytest.mark.parametrize(("invert", "coset"), [(False, None), (True, None), (False, 5), (True, 5)])
def test_emulated_split_ntt_equals_one_piece(parts, invert, coset):
    n = max(parts * parts, 64)
    x = co.to_mont(co.FR, wl.uniform_fr(parts + 3, n))
    m = n // parts
    gens = [sharded.ntt_rank(_t(x[r * m:(r + 1) * m]), parts, r, invert=invert, coset=coset, ops=OracleOps())
            for r in range(parts)]
    got = _assemble_cyclic(sharded.run_emulated(gens))
    assert np.array_equal(got, co.ntt(x, invert=invert, coset=coset))


def test_cyclic_to_block_and_shard_bounds():
    parts, m = 4, 16
    full = np.arange(parts * m * 4, dtype=np.uint64).reshape(parts * m, 4)
    cyclic = [_t(full[t::parts]) for t in range(parts)]
    blocks = sharded.run_emulated([sharded.cyclic_to_block_rank(y, parts, t) for t, y in enumerate(cyclic)])
    assert np.array_equal(np.concatenate([_np(b) for b in blocks]), full)
    assert [sharded.shard_bounds(10, 3, r) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    with pytest.raises(ValueError, match="power of 2"):
        next(sharded.ntt_rank(_t(full[:10]), 3, 0, ops=OracleOps()))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n = 64
    x = co.to_mont(co.FR, wl.uniform_fr(17, n))
    m = n // world
    y = sharded.run_distributed(sharded.ntt_rank(_t(x[rank * m:(rank + 1) * m]), world, rank, coset=5,
                                                 ops=OracleOps()))
    yb = sharded.run_distributed(sharded.cyclic_to_block_rank(y, world, rank))
    # MSM: each rank its slice of 40 points
    pts = co.mul_generator(wl.base_scalars(18, 40))
    sc = wl.skewed_scalars(19, 40)
    lo, hi = sharded.shard_bounds(40, world, rank)
    total = sharded.run_distributed(sharded.msm_rank(_t(pts[lo:hi]), _t(sc[lo:hi]), window_size=5, ops=OracleOps()))
    dist.destroy_process_group()
    out.put((rank, _np(yb).copy(), total))


def test_two_gloo_ranks_split_ntt_and_msm():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted((q.get(timeout=240) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n = 64
    x = co.to_mont(co.FR, wl.uniform_fr(17, n))
    want = co.ntt(x, coset=5)
    assert np.array_equal(np.concatenate([r[1] for r in results]), want)  # block layout after the move
    pts = co.mul_generator(wl.base_scalars(18, 40))
    sc = wl.skewed_scalars(19, 40)
    one = co.msm(pts, sc, 5)
    want_pt = None if one[8] else tuple(_to_ints(one[:8].reshape(2, 4)))
    assert results[0][2] == results[1][2] == want_pt
