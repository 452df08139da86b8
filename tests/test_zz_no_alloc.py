"""
zkb_msm_no_alloc: the MSM entry point for callers that cannot allocate device
memory at call time (a plugin inside a framework that owns all device memory
through its own allocator, or a serving loop that must never reach
cudaMalloc, which can stall every stream on the device). It works in a fixed
scratch array inside the library instead of a caller-provided workspace.

Checked through the C ABI against zkb_msm with a workspace: two calls in a
row on different inputs (the second call reuses the array the first one
left behind), the compact plan the entry point falls back to when the
default plan would not fit the array (at the default and at an explicit
window), and the refusal of a problem larger than the fixed scratch, made
with real device buffers so that a regression shows up as a wrong status
and never as a read through a bad pointer. The results are exact integers,
so they must match bit for bit. This file is collected last, and it also
passes on its own in a fresh process.
"""

from __future__ import annotations

import numpy as np
import pytest

from zkgpu import _native, curve_gpu
from zkgpu import workloads as wl

pytestmark = pytest.mark.gpu

CAPACITY = 64 << 20


def _with_workspace(lib, bases, scalars, n: int, w: int):
    import torch

    ws_bytes = lib.zkb_msm_workspace_bytes(n, w)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    out = torch.empty(16, dtype=torch.int64, device="cuda")
    _native.check(lib.zkb_msm(bases.data_ptr(), scalars.data_ptr(), n, w, out.data_ptr(), ws.data_ptr(),
                              ws_bytes, _native.stream_ptr()))
    return out[:9].cpu().numpy().view(np.uint64)


def _no_alloc(lib, bases, scalars, n: int, w: int):
    import torch

    out = torch.full((16,), -1, dtype=torch.int64, device="cuda")
    _native.check(lib.zkb_msm_no_alloc(bases.data_ptr(), scalars.data_ptr(), n, w, out.data_ptr(),
                                       _native.stream_ptr()))
    return out[:9].cpu().numpy().view(np.uint64)


def test_no_alloc_msm_matches_the_workspace_msm_twice_in_a_row():
    import torch

    lib = _native.lib()
    n = 1 << 16
    # the default plan at 2^16 points needs more than the fixed scratch, so these
    # calls run the compact plan (longer bucket runs, four-bucket segments)
    assert lib.zkb_msm_workspace_bytes(n, 0) > lib.zkb_msm_no_alloc_capacity()
    bases = curve_gpu.mul_generator(wl.base_scalars(61, n))
    first = torch.from_numpy(wl.uniform_fr(62, n)).cuda()
    second = torch.from_numpy(wl.skewed_scalars(63, n)).cuda()
    got1 = _no_alloc(lib, bases, first, n, 0)
    got2 = _no_alloc(lib, bases, second, n, 0)  # reuses the scratch the first call left
    assert np.array_equal(got1, _with_workspace(lib, bases, first, n, 0))
    assert np.array_equal(got2, _with_workspace(lib, bases, second, n, 0))
    assert not np.array_equal(got1, got2)
    assert got1[8] == 0 and got2[8] == 0  # finite points


@pytest.mark.parametrize("n, w", [(80_000, 14), (98_304, 0)])
def test_no_alloc_msm_compact_plan_near_the_capacity(n, w):
    """Sizes whose default plan exceeds the array while the compact plan just fits."""
    import torch

    lib = _native.lib()
    assert lib.zkb_msm_workspace_bytes(n, w) > lib.zkb_msm_no_alloc_capacity()
    bases = curve_gpu.mul_generator(wl.base_scalars(64, n))
    scalars = torch.from_numpy(wl.uniform_fr(65, n)).cuda()
    got = _no_alloc(lib, bases, scalars, n, w)
    assert np.array_equal(got, _with_workspace(lib, bases, scalars, n, w))
    again = _no_alloc(lib, bases, scalars, n, w)
    assert np.array_equal(again, got)


def test_no_alloc_msm_refuses_problems_beyond_its_scratch():
    import torch

    lib = _native.lib()
    cap = lib.zkb_msm_no_alloc_capacity()
    assert cap == CAPACITY
    n = 1 << 20
    assert lib.zkb_msm_workspace_bytes(n, 0) > cap
    # real buffers of the refused size: the call must refuse before any kernel runs
    bases = torch.zeros((n, 2, 4), dtype=torch.int64, device="cuda")
    scalars = torch.zeros((n, 4), dtype=torch.int64, device="cuda")
    out = torch.full((16,), -1, dtype=torch.int64, device="cuda")
    status = lib.zkb_msm_no_alloc(bases.data_ptr(), scalars.data_ptr(), n, 0, out.data_ptr(),
                                  _native.stream_ptr())
    assert status == _native.ZKB_EWORKSPACE
    assert "fixed" in _native.last_error() and "scratch" in _native.last_error()
    torch.cuda.synchronize()
    assert bool((out == -1).all())  # nothing was written
