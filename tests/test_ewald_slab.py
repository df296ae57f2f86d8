"""Ewald k-space slab geometry (slab_normal_axis, slab_lz) and the dipole
term (epsilon_dipole) of the reference's Electrostatic_ewald_k
(electrostatic_ewald_k.cpp:87-126, 197-223; initialize.cpp:49-115).

GPU: forces of 300 ions match the unmodified reference's
(tests/golden/ref_ewald_slab300.npz) with z non-periodic + slab_lz 30 +
epsilon_dipole 0, and with all axes periodic + epsilon_dipole 1; a 10-step
slab run matches; the once-only dipole mode differs from the reference's
per-k-vector accumulation by exactly (n_k - 1) q_i E / m_i.
"""
import os

import numpy as np
import pytest

from caviar_b200 import workloads as W
from helpers import GOLDEN, force_errors


def slab_system(periodic_z):
    s = W.random_ions(300, 10.0, 21, rc=4.0, coef=1.03, kmax=4, alpha=0.8)
    s.bc = (1, 1, 1 if periodic_z else 0)
    return s


def make(cuda_lib, name, prec, mode=None):
    s = slab_system(name != "slab")
    sim = cuda_lib.Simulation(s, precision=prec, policy=cuda_lib.REBUILD_REFERENCE)
    mode = cuda_lib.DIPOLE_REFERENCE if mode is None else mode
    if name == "slab":
        sim.set_ewald_k_geometry(2, 30.0, mode, 0.0)
    else:
        sim.set_ewald_k_geometry(-1, 1.0, mode, 1.0)
    return s, sim


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["slab", "dipole"])
@pytest.mark.parametrize("prec,tol", [(1, 1e-11), (0, 1e-5)])
def test_forces_match_reference(cuda_lib, name, prec, tol):
    d = np.load(os.path.join(GOLDEN, "ref_ewald_slab300.npz"))
    s, sim = make(cuda_lib, name, prec)
    acc, _ = sim.compute_forces()
    assert force_errors(acc, d[f"{name}_acc"])[0] < tol


@pytest.mark.gpu
def test_slab_run_matches_reference(cuda_lib):
    d = np.load(os.path.join(GOLDEN, "ref_ewald_slab300.npz"))
    s, sim = make(cuda_lib, "slab", 1)
    sim.run(10)
    pos, vel, _ = sim.state()
    dp = pos - d["slab_run_pos"]
    dp[:, :2] -= s.box[:2] * np.round(dp[:, :2] / s.box[:2])
    assert np.abs(dp).max() < 1e-9
    assert np.abs(vel - d["slab_run_vel"]).max() < 1e-8


@pytest.mark.gpu
def test_dipole_once_mode(cuda_lib):
    s, ref = make(cuda_lib, "dipole", 1)
    a_ref, _ = ref.compute_forces()
    _, once = make(cuda_lib, "dipole", 1, mode=cuda_lib.DIPOLE_ONCE)
    a_once, _ = once.compute_forces()
    q = s.charge[s.type]
    L = s.box
    pos = s.pos - L * np.floor((s.pos - s.lo) / L)
    M = (q[:, None] * pos).sum(axis=0)
    E = -M * 4 * np.pi / np.prod(L) / (1 + 2 * 1.0)
    nk = 8 ** 3
    expect = a_ref - (nk - 1) * q[:, None] * E[None, :] / s.mass[s.type][:, None]
    assert np.abs(a_once - expect).max() < 1e-9 * np.abs(a_ref).max()
