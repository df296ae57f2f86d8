"""NVE energy conservation over 10^4 steps, against the reference's own.

tests/golden/nve_lj500.json holds the reference's total energy every 1000
steps of a 500-atom LJ fluid (the unmodified reference run by
tests/golden/make_golden.py).  The GPU path runs the same 10^4 steps in both
precisions; its largest deviation of the total energy from the start must be
no worse than the reference's, up to a factor 2 for the trajectory-to-
trajectory spread of a fluctuating quantity (same integrator and time step,
different rounding, so the trajectories decorrelate).
"""
import json
import os

import numpy as np
import pytest

from caviar_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nve_lj500.json")


def test_fixture_is_the_stated_system():
    g = json.load(open(GOLDEN))
    s = W.fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)
    assert g["n"] == s.n == 500 and len(g["total_energy"]) == 11 and g["steps_per_record"] == 1000
    e = np.array(g["total_energy"])
    assert abs(np.abs(e - e[0]).max() / s.n - g["max_abs_dev_per_atom"]) < 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_nve_drift_1e4_steps(cuda_lib, prec):
    g = json.load(open(GOLDEN))
    s = W.fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)
    sim = cuda_lib.Simulation(s, precision=prec)
    _, sc = sim.compute_forces()
    e = [sc["ke"] + sc["e_lj"]]
    th = sim.run(10000, thermo_every=1000)
    for rec in th:
        d = dict(zip(cuda_lib.TH_KEYS, rec))
        e.append(d["ke"] + d["e_lj"])
    e = np.array(e)
    dev = float(np.abs(e - e[0]).max() / s.n)
    assert len(e) == 11
    assert dev <= 2.0 * g["max_abs_dev_per_atom"], (dev, g["max_abs_dev_per_atom"])
    # no systematic drift: the last 5 records' mean stays within the same bound
    assert abs(e[-5:].mean() - e[0]) / s.n <= 2.0 * g["max_abs_dev_per_atom"]
