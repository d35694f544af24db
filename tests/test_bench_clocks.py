"""bench.py's clock summary: the median SM clock under load ignores the
samples taken while the GPU idled between phases; event reasons from every
sample."""
import bench


def test_clock_summary_under_load():
    lines = ["1965, 1965, 900.1, Not Active, Not Active, Not Active, Active, 100",
             "645, 1965, 120.0, Not Active, Not Active, Not Active, Not Active, 0",
             "645, 1965, 118.0, Not Active, Not Active, Not Active, Not Active, 3",
             "1950, 1965, 950.0, Not Active, Not Active, Not Active, Not Active, 98",
             "not a sample"]
    c = bench.summarize_clocks(lines)
    assert c["samples"] == 4 and c["samples_under_load"] == 2
    assert c["sm_mhz"] == 1957.5 and c["sm_mhz_all_samples"] == 1297.5
    assert c["sm_max_mhz"] == 1965.0 and c["reasons"] == ["sw_power_cap"]


def test_clock_summary_without_utilization_column():
    c = bench.summarize_clocks(["1800, 1965, 500, Not Active, Active, Not Active, Not Active"])
    assert c["sm_mhz"] == 1800.0 and c["samples_under_load"] == 0
    assert c["reasons"] == ["hw_thermal_slowdown"]
