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


def test_committed_profile_figures_parse():
    # the roofline line of the headline reads these per-event figures from
    # the committed ncu summaries
    req = bench.ncu_figure(bench.PROFILE_REQUESTS, "requested_bytes_per_event")
    dram = bench.ncu_figure(bench.PROFILE_REQUESTS, "dram_bytes_per_event")
    slab = bench.ncu_traffic_per_event()
    assert req is not None and req > 104          # more than the queue state alone
    assert dram is not None and 0 < dram < req + 1000
    assert slab is not None and slab > 0
    assert bench.ncu_figure(bench.PROFILE_REQUESTS, "no_such_key") is None
    assert bench.ncu_figure("no_such_profile.md", "requested_bytes_per_event") is None


def test_uncertainty_summaries():
    # unc^2 * histories is the per-history relative variance; histories for
    # 1 % divide it by 1e-4; non-finite columns are left out
    unc = np.array([0.1, 0.2, np.nan])
    nh = np.array([1e4, 2.5e3, 1e3])
    s = bench.unc_summary(unc, nh, 1e6)
    assert s["beamlets"] == 2
    assert np.isclose(s["rel_var_x_histories"], 100.0)
    assert np.isclose(s["histories_to_1pct_per_beamlet"], 1e6)
    assert np.isclose(s["seconds_to_1pct_per_beamlet"], 1.0)
    assert np.isclose(s["mean_rel_unc_gt50pct_dmax"], 0.15)
    res = [{"nhist": 1e4, "loop_s": 0.5, "unc": 0.1}, {"nhist": 3e4, "loop_s": 1.5, "unc": 0.1}]
    r = bench.ref_summary(res)
    assert np.isclose(r["value"], 2e4) and np.isclose(r["loop_s"], 2.0)
    assert r["p50_ms"] == 1000.0 and r["unc"]["beamlets"] == 2
