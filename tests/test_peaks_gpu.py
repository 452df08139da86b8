"""
The measured integer issue rates behind the rooflines (zkb_measure_int_peaks):
loops of mad.lo.u32, mad.wide.u32 and the library's Montgomery product, timed
by the SMs' cycle counters and by CUDA events. The checks are plausibility
bounds for a Blackwell SM, not exact values: the measured rates are what the
benchmark divides by.
"""

from __future__ import annotations

import pytest

from zkgpu import _native

pytestmark = pytest.mark.gpu


def test_measured_integer_rates_are_plausible():
    import torch

    p = _native.measure_int_peaks()
    assert p["sms"] == torch.cuda.get_device_properties(0).multi_processor_count
    # four sub-partitions per SM; the low-half multiply-add may issue on more than one pipe,
    # so anything from a half-rate pipe to two full ones is plausible
    assert 32.0 < p["madlo_per_clk_sm"] <= 130.0, p
    # a 32 x 32 -> 64-bit multiply-add issues at most as fast as the low half alone
    assert 8.0 < p["madwide_per_clk_sm"] <= p["madlo_per_clk_sm"] * 1.05, p
    # a 256-bit Montgomery product is at least 128 wide multiply-adds
    assert 0.05 < p["montmul_per_clk_sm"] < p["madwide_per_clk_sm"] / 128 * 1.2, p
    for key in ("madlo_mhz", "madwide_mhz", "montmul_mhz"):
        assert 300.0 < p[key] < 2500.0, (key, p)
