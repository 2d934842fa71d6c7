"""Host logic of bench.py that needs no GPU: the clock summary and the algorithmic byte count."""
import bench


def _row(sm, mx, *reasons):
    # index, clocks.sm, clocks.max.sm, power.draw, active mask, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
    return ["0", str(sm), str(mx), "700.0", "0x0"] + list(reasons)


def test_clock_summary_median_and_reasons():
    cs = bench.ClockSampler(0)
    cs.rows = [
        _row(1965, 1965, "Not Active", "Not Active", "Not Active", "Not Active"),
        _row(1800, 1965, "Not Active", "Not Active", "Not Active", "Active"),
        _row(1900, 1965, "Not Active", "Not Active", "Not Active", "Not Active"),
        ["garbage"],
    ]
    s = cs.summary()
    assert s["sm_mhz"] == 1900 and s["sm_max_mhz"] == 1965 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_reports_thermal_and_hardware_slowdowns():
    cs = bench.ClockSampler(0)
    cs.rows = [_row(1200, 1965, "Active", "Not Active", "Active", "Not Active")]
    assert cs.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_clock_summary_without_samples():
    s = bench.ClockSampler(0).summary()
    assert s["sm_mhz"] is None and s["samples"] == 0 and s["reasons"] == []


def test_algorithmic_bytes_of_the_benchmark_grid():
    """B_apply = S*[T + 2*N_vec + NxNy*Nz] at 128x128x32: the figures the roofline is quoted with."""
    assert bench._algorithmic_bytes(128, 128, 32, 16) == 1_149_239_296
    assert bench._algorithmic_bytes(128, 128, 32, 8) == 574_619_648
    # the tensor alone (T*S, the contraction's algorithmic bytes): 4 packed symmetric + 2 full blocks per unit
    T = 128 * 128 * (4 * 32 * 33 // 2 + 2 * 32 * 32)
    assert T * 16 == 1_090_519_040
