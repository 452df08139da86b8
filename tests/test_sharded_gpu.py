"""
The split NTT and MSM on the GPU (zkgpu.sharded with the library's
arithmetic): G ranks emulated in one process on one GPU (every exchange done
in memory, the per-rank kernels run for real: zkb_ntt_cross_step, zkb_ntt,
zkb_msm), against the one-piece BN254_FR.ntt / msm_pippenger_rows, which the
other test files pin to the reference; the cross-rank kernel also directly
against its Python-integer restatement.
"""

from __future__ import annotations

import numpy as np
import pytest

from zkgpu import curve_gpu, sharded
from zkgpu import workloads as wl
from zkgpu.field256_gpu import BN254_FR
from zkgpu.msm_gpu import msm_pippenger_rows

pytestmark = pytest.mark.gpu


def _split_ntt(x, parts, invert, coset):
    n = int(x.shape[0])
    m = n // parts
    gens = [sharded.ntt_rank(x[r * m:(r + 1) * m], parts, r, invert=invert, coset=coset) for r in range(parts)]
    return sharded.run_emulated(gens)


@pytest.mark.parametrize("parts", [2, 4, 8, 16])
@pytest.mark.parametrize("log_n", [8, 14, 20])
def test_split_ntt_equals_one_piece(parts, log_n):
    import torch

    x = BN254_FR.to_montgomery(wl.uniform_fr(log_n + parts, 1 << log_n))
    for invert, coset in ((False, None), (True, None), (False, 5), (True, 5)):
        ys = _split_ntt(x, parts, invert, coset)
        want = BN254_FR.ntt(x, invert=invert, coset=coset)
        for t, y in enumerate(ys):
            assert bool((y == want[t::parts]).all()), (parts, log_n, invert, coset, t)
        blocks = sharded.run_emulated([sharded.cyclic_to_block_rank(y, parts, t) for t, y in enumerate(ys)])
        assert bool((torch.cat(blocks) == want).all())


def test_cross_kernel_matches_its_restatement():
    from test_sharded import OracleOps, _np

    n = 256
    x = BN254_FR.to_montgomery(wl.uniform_fr(3, n))
    gpu, cpu = sharded.GpuOps(), OracleOps()
    for parts in (2, 4, 8, 16):
        rows = x[: n // parts]  # (G, c) blocks of c = n / G^2 rows
        for part in (0, parts - 1):
            for invert, coset in ((False, None), (True, 7), (False, 7)):
                got = gpu.cross_step(rows, n, parts, part, invert, coset)
                want = cpu.cross_step(rows.cpu(), n, parts, part, invert, coset)
                assert np.array_equal(_np(got.cpu()), _np(want)), (parts, part, invert, coset)


@pytest.mark.parametrize("parts", [2, 4])
def test_split_msm_equals_one_piece(parts):
    n = 5000
    bases = curve_gpu.mul_generator(wl.base_scalars(11, n))
    sc = wl.skewed_scalars(12, n)
    import torch

    sct = torch.from_numpy(sc).cuda()
    gens = []
    for r in range(parts):
        lo, hi = sharded.shard_bounds(n, parts, r)
        gens.append(sharded.msm_rank(bases[lo:hi], sct[lo:hi]))
    got = sharded.run_emulated(gens)
    want = msm_pippenger_rows(bases, sc)
    assert all(g == want for g in got)
