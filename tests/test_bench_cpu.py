"""CPU checks of bench.py's reporting helpers (no GPU): the roofline's
traffic figure comes from the committed pair-kernel profile, the clock record
summarises samples taken during the timed region, and the roofline peak is
the measured one when the measured-peaks file is present."""
import json
import os

import bench


def test_pair_profile_traffic_is_parsed():
    t = bench.profiled_traffic("pair_lj1m.txt")
    # DRAM bytes of one pair-kernel launch on the 1M-atom workload: at least
    # the algorithmic list bytes (4 B x ~76 entries x 1,048,576 atoms)
    assert t is not None and 3.0e8 < t < 5.0e8


def test_clock_summary_from_samples():
    c = bench.Clocks(0)
    c.samples = [(1965.0, []), (1950.0, ["sw_power_cap"]), (1965.0, [])]
    c.mx = 1965.0
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3
    c.samples = []
    assert c.summary() is None


def test_measured_peak_is_used_when_present():
    peak, kind = bench.measured_peaks()
    path = os.path.join(bench.ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            assert kind == "measured" and peak == float(json.load(f)["hbm_gbs"])
    else:
        assert kind == "fallback" and peak > 0
