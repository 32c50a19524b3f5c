"""Host-side helpers of bench.py: the clock record of the timed region (median SM clock,
throttle reasons seen while the steps ran), the committed ncu traffic figure and the
peak bandwidth (no GPU needed)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class _Proc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def _row(sm, reasons=("Not Active",) * 4, mx="1965"):
    return ["0", str(sm), mx, "900.0", "0x0"] + list(reasons)


def test_clock_record_keeps_the_timed_region():
    s = bench.ClockSampler(0)
    s.proc = _Proc()
    s.t0, s.t1 = 10.0, 20.0
    s.rows = [(5.0, _row(900, ("Active", "Not Active", "Not Active", "Not Active"))),  # before: ignored
              (11.0, _row(1965)), (12.0, _row(1950)), (13.0, _row(1320, ("Not Active",) * 3 + ("Active",))),
              (25.0, _row(800, ("Not Active", "Active", "Not Active", "Not Active")))]  # after: ignored
    rec = s.stop()
    assert rec["sm_mhz"] == 1950.0
    assert rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap"]
    assert rec["samples"] == 3


def test_clock_record_without_nvidia_smi():
    s = bench.ClockSampler(0)
    assert s.stop()["reasons"] == ["nvidia-smi unavailable"]


def test_committed_traffic_and_peak():
    t = bench.profile_traffic("jet4400x640")
    assert t is not None and t > 170 * 4400 * 640  # above the algorithmic bytes of a launch
    peak, kind = bench.measured_peaks()
    assert peak > 1000.0 and kind in ("measured", "fallback")


def test_replica_throughput_counts_every_rank():
    # 4 steps of 1000 points on 2 ranks in 2 ms (max over ranks): 4e6 updates/s
    assert bench.replica_throughput(1000, 4, 2, 2.0) == 4e6
