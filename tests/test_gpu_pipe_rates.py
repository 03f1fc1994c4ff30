"""svpf_measure_pipe_rates: the MUFU and FP32 results per SM clock that the
bench's pair roofline divides by, measured on the device.  B200 nominal: 16
MUFU and 128 FP32 results per clock per SM; the measured rates must lie near
them (a rate far off means the calibration kernel does not measure the pipe)."""
import pytest

pytestmark = pytest.mark.gpu


def test_measured_pipe_rates_are_near_nominal(pkg):
    r = pkg.pipe_rates()
    assert 12.0 <= r["mufu_per_clk_sm"] <= 17.0, r
    assert 96.0 <= r["fp32_per_clk_sm"] <= 136.0, r
    assert r["pairs_per_clk_sm"] == min(r["mufu_per_clk_sm"] / 2.0, r["fp32_per_clk_sm"] / 13.0)


def test_rates_repeat(pkg):
    a, b = pkg.pipe_rates(), pkg.pipe_rates()
    assert abs(a["mufu_per_clk_sm"] - b["mufu_per_clk_sm"]) <= 0.02 * a["mufu_per_clk_sm"]
    assert abs(a["fp32_per_clk_sm"] - b["fp32_per_clk_sm"]) <= 0.02 * a["fp32_per_clk_sm"]
