"""
oracle.c_oracle — ctypes wrapper of oracle/libzk_oracle.so (zk_oracle.c).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py). NumPy in, NumPy out:
rows are (n, 4) / (n, 3, 4) / (n, 2, 4) uint64 arrays in the reference's
layout. build() compiles the library with oracle/Makefile when it is missing
or older than its source.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libzk_oracle.so"
SRC = HERE / "zk_oracle.c"

FR, FQ = 0, 1

_lib: ctypes.CDLL | None = None


def build() -> Path:
    if not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        handle = ctypes.CDLL(os.fspath(LIB))
        vp, i64, ci = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        for name in ("zo_field_mul", "zo_field_add", "zo_field_sub"):
            getattr(handle, name).argtypes = [ci, vp, vp, vp, i64]
        for name in ("zo_to_mont", "zo_from_mont"):
            getattr(handle, name).argtypes = [ci, vp, vp, i64]
        handle.zo_ntt.argtypes = [vp, vp, i64, ci, vp, ci, ci, ci]
        handle.zo_ntt.restype = ci
        for name in ("zo_g1_add", "zo_g1_add_affine"):
            getattr(handle, name).argtypes = [vp, vp, vp, i64]
        handle.zo_g1_double.argtypes = [vp, vp, i64]
        handle.zo_g1_to_affine.argtypes = [vp, vp, i64]
        handle.zo_g1_mul_generator.argtypes = [vp, vp, i64, ci]
        handle.zo_msm_window_sums.argtypes = [vp, vp, i64, ci, ci, ci, ci, vp]
        handle.zo_msm_window_sums.restype = ci
        handle.zo_msm.argtypes = [vp, vp, i64, ci, ci, vp]
        handle.zo_msm.restype = ci
        _lib = handle
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _rows(a: np.ndarray, inner: tuple[int, ...]) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    assert a.shape[1:] == inner, a.shape
    return a


def field_op(op: str, fid: int, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a, b = _rows(a, (4,)), _rows(b, (4,))
    out = np.empty_like(a)
    getattr(lib(), f"zo_field_{op}")(fid, _p(a), _p(b), _p(out), a.shape[0])
    return out


def to_mont(fid: int, plain: np.ndarray) -> np.ndarray:
    plain = _rows(plain, (4,))
    out = np.empty_like(plain)
    lib().zo_to_mont(fid, _p(plain), _p(out), plain.shape[0])
    return out


def from_mont(fid: int, rows: np.ndarray) -> np.ndarray:
    rows = _rows(rows, (4,))
    out = np.empty_like(rows)
    lib().zo_from_mont(fid, _p(rows), _p(out), rows.shape[0])
    return out


def ntt(rows: np.ndarray, *, invert: bool = False, coset: int | None = None, threads: int = 1,
        stages: tuple[int, int] = (0, 64)) -> np.ndarray:
    """NTT over BN254 Fr of Montgomery rows (zkgpu/ntt.py's algorithm); stages limits the
    butterfly stages run (for timing a sample)."""
    rows = _rows(rows, (4,))
    out = np.empty_like(rows)
    g = None
    if coset is not None:
        g = np.array([(coset >> (64 * j)) & (2**64 - 1) for j in range(4)], dtype=np.uint64)
    rc = lib().zo_ntt(_p(rows), _p(out), rows.shape[0], int(invert), None if g is None else _p(g),
                      threads, stages[0], stages[1])
    if rc != 0:
        raise ValueError(f"bad NTT size {rows.shape[0]}")
    return out


def g1_op(op: str, a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    a = _rows(a, (3, 4))
    out = np.empty_like(a)
    if op == "double":
        lib().zo_g1_double(_p(a), _p(out), a.shape[0])
    else:
        b = _rows(b, (3, 4) if op == "add" else (2, 4))
        getattr(lib(), f"zo_g1_{op}")(_p(a), _p(b), _p(out), a.shape[0])
    return out


def g1_to_affine(a: np.ndarray) -> np.ndarray:
    """(n, 9): plain x limbs, y limbs, infinity flag."""
    a = _rows(a, (3, 4))
    out = np.empty((a.shape[0], 9), dtype=np.uint64)
    lib().zo_g1_to_affine(_p(a), _p(out), a.shape[0])
    return out


def mul_generator(k: np.ndarray, threads: int = 1) -> np.ndarray:
    """(n, 2, 4) affine Montgomery rows of k_i G for plain scalars k (n, 4) in [1, r)."""
    k = _rows(k, (4,))
    out = np.empty((k.shape[0], 2, 4), dtype=np.uint64)
    lib().zo_g1_mul_generator(_p(k), _p(out), k.shape[0], threads)
    return out


def msm(points: np.ndarray, scalars: np.ndarray, w: int, threads: int = 1) -> np.ndarray:
    """The reference's Pippenger at window w: (9,) plain x, y limbs and an infinity flag."""
    points, scalars = _rows(points, (2, 4)), _rows(scalars, (4,))
    out = np.empty(9, dtype=np.uint64)
    rc = lib().zo_msm(_p(points), _p(scalars), points.shape[0], w, threads, _p(out))
    if rc != 0:
        raise ValueError("bad MSM arguments")
    return out


def msm_window_sums(points: np.ndarray, scalars: np.ndarray, w: int, win_lo: int, win_hi: int,
                    threads: int = 1) -> np.ndarray:
    """Window sums win_lo..win_hi-1 of the reference's Pippenger, Jacobian Montgomery rows."""
    points, scalars = _rows(points, (2, 4)), _rows(scalars, (4,))
    out = np.empty((win_hi - win_lo, 3, 4), dtype=np.uint64)
    rc = lib().zo_msm_window_sums(_p(points), _p(scalars), points.shape[0], w, win_lo, win_hi,
                                  threads, _p(out))
    if rc != 0:
        raise ValueError("bad MSM arguments")
    return out
