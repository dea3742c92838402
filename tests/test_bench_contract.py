"""bench.py's command-line defaults and the pieces of its JSON line that need no GPU: one GPU
and at least 3 warm-up steps by default, the workload names and sizes, and the clock
record (median SM clock under load and the NVML clock-event reasons seen while timing)."""
import sys

import bench


def _parse(*args):
    old = sys.argv
    sys.argv = ["bench.py", *args]
    try:
        return bench.parse()
    finally:
        sys.argv = old


def test_defaults_are_one_gpu_and_three_warmup_steps():
    a = _parse()
    assert (a.gpus, a.warmup, a.impl, a.workload, a.level, a.precision) == (1, 3, "ours", "catchment", 12, 32)
    assert a.steps >= 100   # a timed window long enough to be sampled (about 0.6 s on the device)
    assert _parse("--workload", "ensemble").steps == 20 and _parse("--steps", "7").steps == 7
    w = bench.workload(a)
    assert "4096^2" in w["workload"] and w["max_ref_lvl"] == 12 and "L2" in w["l2"]


def test_decode_defaults_to_the_reference_decode():
    a = _parse()
    assert a.decode == "reference" and bench.workload(a)["decode"] == "reference"
    assert bench.workload(_parse("--decode", "keep"))["decode"] == "keep"


def test_urban_workload_defaults_to_8192():
    a = _parse("--workload", "urban")
    assert a.level == 13
    assert "8192^2" in bench.workload(a)["workload"]
    assert _parse("--workload", "urban", "--level", "11").level == 11


def test_clock_record_median_and_reasons():
    c = bench.Clocks(0)
    assert c.summary()["reasons"] == ["unsampled"]
    # (SM MHz, max SM MHz, NVML clock-event reason bits): power cap (0x4) on one sample,
    # hardware slowdown (0x8) on another, idle (0x1) is not a reason that rejects a run
    c.rows = [(1965.0, 1965.0, 0x0), (1900.0, 1965.0, 0x4), (1965.0, 1965.0, 0x8 | 0x1)]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
