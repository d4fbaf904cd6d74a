"""The bench's clock record: nvidia-smi samples (every 20 ms, with their
times) summarised as the median and maximum SM clock and the throttle
reasons seen, plus the count and lowest clock of the samples that fall in
the timed window."""
import datetime

import bench


def _line(t, sm, power_cap="Not Active"):
    ts = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    return "%s, 0, %s, 1965, 700.5, 0x0000000000000000, Not Active, Not Active, Not Active, %s\n" % (
        ts, sm, power_cap)


def test_summary_of_the_samples_and_of_the_timed_window():
    t0 = 1_800_000_000.0
    lines = [_line(t0 + 0.02 * i, 1965) for i in range(10)]
    lines += [_line(t0 + 0.20 + 0.02 * i, sm) for i, sm in enumerate((1965, 1800, 1965))]
    lines += [_line(t0 + 0.30, 1965, power_cap="Active"), "garbage line\n"]
    out = bench.ClockSampler.summarize(lines, window=(t0 + 0.19, t0 + 0.25))
    assert out["samples"] == 14 and out["interval_ms"] == 20
    assert out["sm_mhz"] == 1965 and out["sm_max_mhz"] == 1965
    assert out["reasons"] == ["sw_power_cap"]
    assert out["timed_samples"] == 3 and out["timed_sm_mhz_min"] == 1800


def test_no_samples_and_no_window():
    assert bench.ClockSampler.summarize([])["reasons"] == ["no samples"]
    out = bench.ClockSampler.summarize([_line(1_800_000_000.0, 1965)])
    assert "timed_samples" not in out and out["sm_mhz"] == 1965
