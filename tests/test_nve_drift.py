"""NVE energy conservation over 10^4 steps, against the reference's own.

tests/golden/nve_lj500.json and nve_ions500.json hold the reference's total
energy every 100 steps over 10^4 velocity-Verlet steps (the unmodified
reference, run by tests/golden/make_golden.py) of a 500-atom LJ fluid and of
500 ions with LJ + Ewald real and k space (the ions start from the
reference's own state after 2000 steps, stored in the record).  The GPU path
runs the same 10^4 steps in both precisions under the reference's rebuild
trigger and records the same energy every 100 steps.

The trajectories decorrelate (same integrator and time step, different
rounding), so the GPU trace is compared with the reference's statistically.
For each trace of 101 records E_k, a least-squares line E = a + b t gives
  * the drift b (per atom per 10^4 steps) and its standard error
    SE = s / sqrt(sum (t - tbar)^2) with s the residual spread, doubled for
    the correlation of neighbouring records;
  * the fluctuation s (per atom).
Bounds: |b_gpu| <= |b_ref| + 3 (SE_gpu + SE_ref), and s_gpu <= 1.5 s_ref (the
spread of 101 correlated samples with at least ~25 independent ones has a
relative standard error of about 14 %, so 1.5 allows more than three).
"""
import json
import os

import numpy as np
import pytest

from caviar_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLDEN, f"nve_{name}.json")) as f:
        return json.load(f)


def system(name, g):
    if name == "lj500":
        return W.fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)
    s = W.random_ions(500, 16.0, seed=13, rc=5.0, kmax=4, alpha=0.6)
    s.pos = np.asarray(g["pos0"], np.float64)
    s.vel = np.asarray(g["vel0"], np.float64)
    return s


def trace_stats(e, n, steps_per_record):
    """(drift per atom per 10^4 steps, its standard error, fluctuation per atom)."""
    e = np.asarray(e, np.float64) / n
    t = np.arange(len(e), dtype=np.float64) * steps_per_record / 1e4
    b, a = np.polyfit(t, e, 1)
    res = e - (a + b * t)
    s = float(np.sqrt(np.sum(res * res) / (len(e) - 2)))
    se = 2.0 * s / float(np.sqrt(np.sum((t - t.mean()) ** 2)))
    return float(b), se, s


@pytest.mark.parametrize("name", ["lj500", "ions500"])
def test_fixture_is_the_stated_system(name):
    g = load(name)
    s = system(name, g)
    assert g["n"] == s.n == 500 and len(g["total_energy"]) == 101 and g["steps_per_record"] == 100
    b, se, sd = trace_stats(g["total_energy"], s.n, 100)
    assert np.isfinite([b, se, sd]).all() and sd > 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("name", ["lj500", "ions500"])
def test_nve_drift_1e4_steps(cuda_lib, name, prec):
    g = load(name)
    s = system(name, g)
    sim = cuda_lib.Simulation(s, precision=prec, policy=cuda_lib.REBUILD_REFERENCE)
    keys = ("ke", "e_lj", "e_ewald_r", "e_ewald_k", "e_self")
    _, sc = sim.compute_forces()
    e = [sum(sc[k] for k in keys)]
    th = sim.run(10000, thermo_every=100)
    for rec in th:
        d = dict(zip(cuda_lib.TH_KEYS, rec))
        e.append(sum(d[k] for k in keys))
    assert len(e) == 101
    b_ref, se_ref, s_ref = trace_stats(g["total_energy"], s.n, 100)
    b, se, sd = trace_stats(e, s.n, 100)
    print(f"{name} prec {prec}: drift {b:.3e} +- {se:.1e} (reference {b_ref:.3e} +- {se_ref:.1e}), "
          f"fluctuation {sd:.3e} (reference {s_ref:.3e})")
    assert abs(b) <= abs(b_ref) + 3.0 * (se + se_ref), (b, se, b_ref, se_ref)
    assert sd <= 1.5 * s_ref, (sd, s_ref)
