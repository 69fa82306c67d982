"""The two calibration kernels whose results are the roofline denominators of bench.py: the
INT32 lane-op rate (analysis kernels) and the FP64 rate (transform kernel). Both must return a
rate in the range a B200 can reach (148 SMs near 2 GHz)."""
import pytest

pytestmark = pytest.mark.gpu


def test_int32_peak_is_plausible(ctx):
    ops = ctx.measure_int32_peak()
    assert 5e12 < ops < 2e14, ops


def test_fp64_peak_is_plausible(ctx):
    flops = ctx.measure_fp64_peak()
    assert 5e12 < flops < 1.5e14, flops
