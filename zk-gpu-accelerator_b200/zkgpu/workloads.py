"""
zkgpu.workloads — seeded synthetic inputs with the shapes of the benchmark configs.

Pure NumPy, deterministic in the seed, so tests, benchmarks and fixture
scripts all regenerate the same inputs:

- uniform_fr(seed, n): (n, 4) uint64 rows of values uniform in [0, r),
  canonical; limb 3 is masked to 62 bits and rows >= r are redrawn.
- skewed_scalars(seed, n): witness-like scalars: 60% in {0, 1}, 20% below
  2^32, 20% uniform in [0, r).
- base_scalars(seed, n): k_i uniform in [1, r), the discrete logs of the base
  points P_i = k_i G (zkgpu.curve_gpu.mul_generator makes the points).
"""

from __future__ import annotations

import numpy as np

# BN254 scalar field r (kept local so this module has no package imports)
R = 21888242871839275222246405745257275088548364400416034343698204186575808495617

_R_LIMBS = np.array([(R >> (64 * j)) & (2**64 - 1) for j in range(4)], dtype=np.uint64)


def _below_r(rows: np.ndarray) -> np.ndarray:
    """Boolean mask of rows whose 256-bit value is below r."""
    lt = np.zeros(rows.shape[0], dtype=bool)
    eq = np.ones(rows.shape[0], dtype=bool)
    for j in range(3, -1, -1):
        lt |= eq & (rows[:, j] < _R_LIMBS[j])
        eq &= rows[:, j] == _R_LIMBS[j]
    return lt


def _uniform_rows(rng: np.random.Generator, n: int) -> np.ndarray:
    out = np.empty((n, 4), dtype=np.uint64)
    filled = 0
    while filled < n:
        need = n - filled
        draw = rng.integers(0, 2**64, size=(need + need // 3 + 16, 4), dtype=np.uint64)
        draw[:, 3] &= np.uint64((1 << 62) - 1)
        ok = draw[_below_r(draw)]
        take = min(need, ok.shape[0])
        out[filled : filled + take] = ok[:take]
        filled += take
    return out


def uniform_fr(seed: int, n: int) -> np.ndarray:
    """(n, 4) uint64 plain rows uniform in [0, r)."""
    return _uniform_rows(np.random.default_rng(seed), n)


def skewed_scalars(seed: int, n: int) -> np.ndarray:
    """(n, 4) uint64 plain rows: 60% in {0, 1}, 20% below 2^32, 20% uniform in [0, r)."""
    rng = np.random.default_rng(seed)
    u = rng.random(n)
    small = rng.integers(0, 2, size=n, dtype=np.uint64)
    mid = rng.integers(0, 2**32, size=n, dtype=np.uint64)
    full = _uniform_rows(rng, n)
    out = np.zeros((n, 4), dtype=np.uint64)
    sel_small = u < 0.6
    sel_mid = (u >= 0.6) & (u < 0.8)
    sel_full = u >= 0.8
    out[sel_small, 0] = small[sel_small]
    out[sel_mid, 0] = mid[sel_mid]
    out[sel_full] = full[sel_full]
    return out


def base_scalars(seed: int, n: int) -> np.ndarray:
    """(n, 4) uint64 plain rows k_i uniform in [1, r) (zero redrawn as 1)."""
    k = uniform_fr(seed, n)
    zero = ~k.any(axis=1)
    k[zero, 0] = 1
    return k


def rows_to_ints(rows: np.ndarray) -> list[int]:
    rows = np.ascontiguousarray(rows, dtype=np.uint64).reshape(-1, 4)
    return [int(r[0]) | int(r[1]) << 64 | int(r[2]) << 128 | int(r[3]) << 192 for r in rows]
