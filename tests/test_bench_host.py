"""Host-side logic of bench.py, without a GPU: the phases of a per-cycle
trace (injection, after the last injection, drain) and the clock record
parsed from nvidia-smi lines (median SM clock, throttle reasons)."""
import numpy as np

import bench


def test_trace_phases_with_and_without_drain():
    rows = [[100, 100, 0, 0.1, 0.2, 0.3],
            [50, 80, 60, 0.1, 0.2, 0.4],
            [0, 10, 70, 0.01, 0.1, 0.5],
            [0, 2, 30, 0.01, 0.05, 0.2],
            [0, 1, 9, 0.0, 0.0, 7.5]]       # the drain
    p = bench.trace_phases(rows)
    assert p["cycles"] == 4 and p["last_injection_cycle"] == 1
    assert np.isclose(p["injection_ms"], 0.6 + 0.7)
    assert np.isclose(p["after_injection_ms"], 0.61 + 0.26)
    assert p["drain_ms"] == 7.5 and p["drain_particles"] == 10
    q = bench.trace_phases(rows[:-1])
    assert q["cycles"] == 4 and q["drain_ms"] == 0.0 and q["drain_particles"] == 0
    assert np.isclose(q["after_injection_ms"], p["after_injection_ms"])


def test_clock_record_median_and_reasons():
    c = bench.ClockSampler(0)
    c.proc = None
    assert c.stop()["reasons"] == ["nvidia-smi unavailable"]

    class Done:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    c.proc = Done()
    c.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1800, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1965, 1965, 800.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "garbage"]
    r = c.stop()
    assert r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0 and r["samples"] == 3
    assert r["reasons"] == ["sw_power_cap"]
