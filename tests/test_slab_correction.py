"""force_field electrostatic_ewald_slab_correction next to the slab Ewald sum
(electrostatic_ewald_slab_correction.cpp and its initialize/field/energy
files).

GPU: forces of 300 ions (periodic in two directions, normal axis z or x)
match the unmodified reference's (tests/golden/ref_slab_correction300.npz),
and a 10-step run (where the reference's one-call-late dipole term enters)
matches too.
"""
import os

import numpy as np
import pytest

from caviar_b200 import workloads as W
from helpers import GOLDEN, force_errors


def make(cuda_lib, axis, prec):
    s = W.random_ions(300, 10.0, 21, rc=4.0, coef=1.03, kmax=4, alpha=0.8)
    s.bc = (0, 1, 1) if axis == 0 else (1, 1, 0)
    sim = cuda_lib.Simulation(s, precision=prec, policy=cuda_lib.REBUILD_REFERENCE)
    sim.set_ewald_k_geometry(axis, 30.0, cuda_lib.DIPOLE_OFF, 0.0)
    sim.set_ewald_slab_correction(axis, 30.0, 4, 4, 1.0)
    return s, sim


@pytest.mark.gpu
@pytest.mark.parametrize("axis,name", [(2, "z"), (0, "x")])
@pytest.mark.parametrize("prec,tol", [(1, 1e-11), (0, 1e-5)])
def test_forces_match_reference(cuda_lib, axis, name, prec, tol):
    d = np.load(os.path.join(GOLDEN, "ref_slab_correction300.npz"))
    _, sim = make(cuda_lib, axis, prec)
    acc, _ = sim.compute_forces()
    assert force_errors(acc, d[f"{name}_acc"])[0] < tol


@pytest.mark.gpu
def test_run_matches_reference(cuda_lib):
    d = np.load(os.path.join(GOLDEN, "ref_slab_correction300.npz"))
    s, sim = make(cuda_lib, 2, 1)
    sim.run(10)
    pos, vel, _ = sim.state()
    dp = pos - d["z_run_pos"]
    dp[:, :2] -= s.box[:2] * np.round(dp[:, :2] / s.box[:2])
    assert np.abs(dp).max() < 1e-9
    assert np.abs(vel - d["z_run_vel"]).max() < 1e-8


@pytest.mark.gpu
def test_rejects_thin_gap(cuda_lib):
    s = W.random_ions(300, 10.0, 21, rc=4.0, coef=1.03, kmax=4, alpha=0.8)
    with pytest.raises(cuda_lib.CvrError):
        sim = cuda_lib.Simulation(s, precision=1)
        sim.set_ewald_slab_correction(2, 5.0, 4, 4, 1.0)  # lz below the box height
