"""bench.py's clock record: the nvidia-smi samples (CLOCK_QUERY, csv without
header or units) are filtered to the timed window by their timestamps, and
the throttle reasons seen there are reported by name.  Host logic only."""
import datetime

import bench


def line(t, sm, power=400.0, reasons=("Not Active",) * 4, max_sm=1965):
    stamp = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    return ", ".join(["0", str(sm), str(max_sm), "%.2f" % power, "0x0000000000000000", *reasons, stamp])


def test_samples_inside_the_window_only():
    t0 = 1_800_000_000.0
    lines = [line(t0 - 1.0, 900, reasons=("Active", "Not Active", "Not Active", "Not Active"))]
    lines += [line(t0 + 0.05 * k, 1965 - k, power=300.0 + k) for k in range(1, 6)]
    lines += [line(t0 + 2.0, 1200, power=900.0)]
    c = bench.Clocks.summarize(lines, t0, t0 + 1.0)
    assert c["samples"] == 5 and c["window"] == "timed region"
    assert c["sm_mhz"] == 1962.0 and c["sm_max_mhz"] == 1965.0 and c["power_w_max"] == 305.0
    assert c["reasons"] == []  # the hw_slowdown sample lies before the window


def test_reasons_by_name():
    t0 = 1_800_000_000.0
    lines = [line(t0 + 0.1, 1500, reasons=("Not Active", "Not Active", "Not Active", "Active")),
             line(t0 + 0.2, 1400, reasons=("Not Active", "Active", "Not Active", "Active"))]
    c = bench.Clocks.summarize(lines, t0, t0 + 1.0)
    assert c["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert c["sm_mhz"] == 1450.0


def test_short_window_takes_the_nearest_samples():
    t0 = 1_800_000_000.0
    lines = [line(t0 - 0.2, 1000), line(t0 - 0.03, 1900), line(t0 + 0.04, 1960), line(t0 + 0.3, 1000)]
    c = bench.Clocks.summarize(lines, t0, t0 + 0.01)  # no sample inside
    assert c["samples"] == 2 and c["sm_mhz"] == 1930.0
    assert c["window"].startswith("nearest samples")


def test_no_samples():
    assert bench.Clocks.summarize([], 0.0, 1.0) is None
    assert bench.Clocks.summarize(["garbage", "0, [N/A], 1965"], 0.0, 1.0) is None
