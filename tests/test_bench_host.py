"""bench.py's host-side bookkeeping without a GPU: the clock record taken from
nvidia-smi samples (busy samples only, throttle reasons by name), percentiles,
the whole-job throughput and the L2 flush buffer."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def row(sm, util, hw="Not Active", cap="Not Active", mx=1965):
    return "0, %s, %s, 512.30, 0x0000000000000000, %s, Not Active, Not Active, %s, %s" % (sm, mx, hw, cap, util)


def sampler(lines):
    c = bench.ClockSampler(None)
    c.out = "\n".join(lines) + "\n"
    return c


def test_clock_summary_uses_busy_samples_and_names_reasons():
    lines = [row(345, 0, hw="Active"),  # idle before the timed work: not counted
             row(1965, 100), row(1965, 98, cap="Active"), row(1950, 100), row(1965, 97),
             row(400, 3)]
    s = sampler(lines).summary()
    assert s["sm_mhz"] == 1965 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == ["sw_power_cap"]
    assert s["samples"] == 6 and s["busy_samples"] == 4


def test_clock_summary_falls_back_to_all_samples_and_tolerates_missing_values():
    s = sampler([row(1200, 10), row("[N/A]", 20), row(1300, 30)]).summary()
    assert s["sm_mhz"] == 1250 and s["busy_samples"] == 0 and s["reasons"] == []
    assert sampler([]).summary()["reasons"] == ["unavailable"]
    assert sampler(["garbage"]).summary()["samples"] == 0


def test_throughput_and_percentiles():
    assert bench.job_throughput(200, 100.0, 4) == pytest.approx(4 * 200 / 0.1)
    assert bench.percentile([1.0, 2.0, 3.0, 4.0], 50) == pytest.approx(2.5)
    assert bench.percentile([], 99) == 0.0


def test_l2_flush_buffer_exceeds_l2_and_fills_with_16_byte_vectors():
    """The flush writes FLUSH_BYTES (twice the 126 MB L2) as float32, the dtype
    whose fill_ stores 16 bytes per thread; a uint8 buffer of the same size
    fills at about half the speed, which the pipelined e2e run would count."""
    import torch
    buf = bench.l2_flush_buffer(torch.device("cpu"))
    assert buf.dtype == torch.float32
    assert buf.numel() * buf.element_size() == bench.FLUSH_BYTES >= 2 * 126 * 10**6
    buf.fill_(7 & 255)
    assert float(buf[-1]) == 7.0
