"""
The autotuner on the GPU (zkgpu.autotune): a measured table for small sizes
is valid, is cached and reloaded under this device's key, and applying it
changes no result: the same NTT rows and MSM points as the built-in rules,
which the other test files pin to the reference.
"""

from __future__ import annotations

import pytest

from zkgpu import _native, autotune, curve_gpu
from zkgpu import workloads as wl
from zkgpu.field256_gpu import BN254_FR
from zkgpu.msm_gpu import msm_pippenger_rows

pytestmark = pytest.mark.gpu


def test_tuned_tables_change_speed_not_results(tmp_path):
    msm_logs, ntt_logs = (10, 12), (10, 12, 16)
    xs = {lg: BN254_FR.to_montgomery(wl.uniform_fr(lg, 1 << lg)) for lg in ntt_logs}
    bases = curve_gpu.mul_generator(wl.base_scalars(5, 1 << 12))
    sc = {lg: wl.uniform_fr(6 + lg, 1 << lg) for lg in msm_logs}
    autotune.clear()
    before_ntt = {lg: BN254_FR.ntt(x, coset=5) for lg, x in xs.items()}
    before_msm = {lg: msm_pippenger_rows(bases[: 1 << lg], s) for lg, s in sc.items()}
    path = tmp_path / "tune.json"
    try:
        table = autotune.autotune(msm_logs, ntt_logs, path=path)
        for lg in msm_logs:
            e = table["msm"][lg]
            assert 1 <= e["window"] <= 20 and e["ms"] > 0
            assert _native.lib().zkb_msm_default_window(1 << lg) == e["window"]
        for lg in ntt_logs:
            e = table["ntt"][lg]
            assert 8 <= e["max_log_radix"] <= 12 and 9 <= e["cta_log_elems"] <= 12
        for lg, x in xs.items():
            assert bool((BN254_FR.ntt(x, coset=5) == before_ntt[lg]).all()), lg
        for lg, s in sc.items():
            assert msm_pippenger_rows(bases[: 1 << lg], s) == before_msm[lg], lg
        # a second call reuses the cache under this device's key
        again = autotune.autotune(msm_logs, ntt_logs, path=path)
        assert {int(k): v["window"] for k, v in again["msm"].items()} == {k: v["window"] for k, v in table["msm"].items()}
        assert again["device"] == autotune.device_key()
    finally:
        autotune.clear()
