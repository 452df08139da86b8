"""
Test configuration: import paths, the `gpu` marker, and fixture helpers.

`-m "not gpu"` runs on any machine: the oracle against the reference's
golden vectors, the host-side logic, and the C ABI's exports. `-m gpu` runs
the parity tests proper on a B200: every GPU result is compared bit-exactly
with the golden fixtures or the oracle. GPU tests are skipped when no CUDA
device is visible.
"""

from __future__ import annotations

import json
import sys
from functools import cache
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "zk-gpu-accelerator_b200"))
sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (NVIDIA B200, sm_100a)")


def _cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device visible")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@cache
def golden(name: str) -> dict:
    return json.loads((GOLDEN / name).read_text())


def h(s: str) -> int:
    return int(s, 16)


def hs(xs: list[str]) -> list[int]:
    return [int(s, 16) for s in xs]
