"""Host-side pieces of bench.py's measurement (no GPU): the clock-record
parsing (only samples taken inside the timed region count) and the roofline
object (algorithmic bytes of the dominant kernel, the measured and the
specification HBM bandwidth, the dominant kernel's measured DRAM traffic,
the atomic ceiling of a scatter)."""
import pytest

import bench


def _line(sm, reasons=("Not Active",) * 4):
    # index, clocks.sm, clocks.max.sm, power.draw, active mask, then the four reasons
    return ", ".join(["0", str(sm), "1965", "700.00", "0x0000000000000000", *reasons]) + "\n"


def test_clock_parse_skips_samples_before_the_timed_region():
    lines = [_line(300), _line(1965), _line(1965), _line(1950)]
    r = bench.ClockSampler.parse(lines, skip=1)
    assert r["samples"] == 3
    assert r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == []


def test_clock_parse_reports_throttle_reasons():
    lines = [_line(1965), _line(1800, ("Not Active", "Not Active", "Not Active", "Active"))]
    r = bench.ClockSampler.parse(lines, skip=0)
    assert r["reasons"] == ["sw_power_cap"]
    r = bench.ClockSampler.parse([_line(1500, ("Active", "Not Active", "Not Active", "Not Active"))])
    assert r["reasons"] == ["hw_slowdown"]


def test_clock_parse_falls_back_to_the_last_sample():
    # the sampler started late: no line after the skip, the last one stands in
    r = bench.ClockSampler.parse([_line(1965)], skip=1)
    assert r["samples"] == 1
    assert bench.ClockSampler.parse([], skip=0) is None
    assert bench.ClockSampler.parse(["garbage\n"], skip=0) is None


KERNEL = "pp_brick_pullbwd_kernel mode=5 order=3 cb=3"


def _ops(pull_bwd_ms):
    return {"pull_fwd": {"avg_ms": 1.0, "total_ms": 20.0},
            "push_fwd": {"avg_ms": 1.4, "total_ms": 28.0},
            "push_bwd": {"avg_ms": 1.0, "total_ms": 20.0},
            "pull_bwd": {"avg_ms": pull_bwd_ms, "total_ms": 20 * pull_bwd_ms, "kernel": KERNEL}}


def test_roofline_of_config2():
    nvox, C = 192 ** 3, 3
    labels = ["pull_fwd", "push_fwd", "push_bwd", "pull_bwd"]
    r = bench.roofline(_ops(2.4), labels, nvox, C, 6.4, None)
    assert r["op"] == "pull_bwd" and r["kernel"] == KERNEL
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    per = (24 + 3 * 4 * C) * nvox
    assert r["algorithmic_bytes_per_launch"] == per
    assert r["achieved"] == pytest.approx(per / 2.4e-3 / 1e9, rel=1e-3)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"], abs=1e-4)
    assert r["spec_gbs"] == 8000.0
    assert r["frac_of_spec"] == pytest.approx(r["achieved"] / 8000.0, abs=1e-4)
    # the dominant kernel's DRAM traffic comes from the ncu capture of the
    # kernel that ran (looked up by its name), null for a kernel not captured
    saved = dict(bench.MEASURED_TRAFFIC)
    try:
        bench.MEASURED_TRAFFIC.clear()
        bench.MEASURED_TRAFFIC[KERNEL] = 5.0e8
        r = bench.roofline(_ops(2.4), labels, nvox, C, 6.4, None)
        assert r["traffic"] == pytest.approx(5.0e8) and KERNEL in r["traffic_source"]
        bench.MEASURED_TRAFFIC.clear()
        r = bench.roofline(_ops(2.4), labels, nvox, C, 6.4, None)
        assert r["traffic"] is None
    finally:
        bench.MEASURED_TRAFFIC.clear()
        bench.MEASURED_TRAFFIC.update(saved)
    # a scatter: the atomic ceiling beside the HBM roofline
    assert r["atomic"]["adds_per_launch"] == 64 * C * nvox
    assert 0 < r["atomic"]["frac"] < 1


def test_roofline_traffic_only_for_the_captured_workload():
    r = bench.roofline(_ops(2.4), ["pull_bwd"], 128 ** 3, 3, 3.0, None)
    assert r["traffic"] is None and r["traffic_source"] is None
    r = bench.roofline(_ops(2.4), ["pull_bwd"], 192 ** 3, 3, 6.4, 1.0e9)
    assert r["traffic"] == 1.0e9 and r["traffic_source"] == "--traffic"


def test_batched_roofline():
    """Algorithmic bytes of the batched step: per volume, points x the chain's
    per-point bytes at the volume's channel count and storage size."""
    import bench
    r = bench.batched_roofline([(10, 20, 30), (5, 5, 5)], [3, 1], 4, 0.002, 2)
    per = sum(bench.algo_bytes(k, 4, 3) for k in ("pull_fwd", "push_fwd", "push_bwd", "pull_bwd")) * 6000
    per += sum(bench.algo_bytes(k, 4, 1) for k in ("pull_fwd", "push_fwd", "push_bwd", "pull_bwd")) * 125
    assert r["algorithmic_bytes_per_step"] == per
    assert r["achieved"] == pytest.approx(per / 2e-6 / 1e9, rel=1e-3)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"], abs=1e-4)
