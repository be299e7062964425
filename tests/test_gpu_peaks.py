"""bem_measure_peaks: the microbenchmarks behind the roofline denominators
run, finish without a device timeout, and land in a plausible range for a
B200 (148 SMs at up to 1965 MHz)."""
import pytest

from bem_mececcs_b200 import capi

pytestmark = pytest.mark.gpu


def test_measured_peaks_plausible():
    ctx = capi.Context(0)
    p = ctx.peaks()
    ctx.close()
    assert 10.0 < p["fp64_fma"] < 80.0
    assert 30.0 < p["fp32_fma"] < 160.0
    assert 10.0 < p["fp64_dmma"] < 80.0
    assert 200.0 < p["tf32_umma_n128"] < 2000.0
    assert 200.0 < p["tf32_umma_n256"] < 2000.0
